// nrldpc_api.cu — the C ABI: reference-compatible entry points and the
// batched device API.  Host code only; kernels live in nrldpc_fixed.cu and
// nrldpc_float.cu.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include <math.h>

#include "nrldpc_bounds.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {

namespace {

uint64_t g_channel_seed = 0x5EEDull;
uint64_t g_channel_calls = 0;

// Channel constants exactly as the reference computes them in float
// (c_lib/tx_rx_process.c:71-97, :298-299).
bool channel_constants(int Qm, float noise_power_db, float* nv, float* sigma, float* A) {
  float k;
  switch (Qm) {
    case 1:
    case 2: k = 2.0f; break;
    case 4: k = 10.0f; break;
    case 6: k = 42.0f; break;
    case 8: k = 170.0f; break;
    default: return false;
  }
  *A = 1.0f / sqrtf(k);
  *nv = powf(10.0f, noise_power_db / 10.0f);
  *sigma = sqrtf(*nv / 2.0f);
  return true;
}

std::atomic<int64_t> g_launches{0};
std::mutex g_mu;

// Default algo-3 table: alpha by check-node degree
// (c_lib/degree_fixedpoint_ldpc_decoder.c:188-222).
const int16_t kDefaultDegreeAlpha[kMaxDegree] = {26623, 26623, 26623, 26623, 24575, 24575, 24575,
                                                 24575, 22527, 22527, 22527, 22527, 22527, 22527,
                                                 22527, 22527, 22527, 22527, 22527};
int16_t g_degree_alpha[kMaxDegree];
bool g_degree_alpha_init = false;

int16_t degree_alpha(int deg) {
  if (!g_degree_alpha_init) {
    memcpy(g_degree_alpha, kDefaultDegreeAlpha, sizeof(g_degree_alpha));
    g_degree_alpha_init = true;
  }
  if (deg <= 0) return g_degree_alpha[0];
  if (deg > kMaxDegree) return g_degree_alpha[kMaxDegree - 1];
  return g_degree_alpha[deg - 1];
}

// Algo-2 tables, [T][rows] packed alpha|beta<<16.  The built-in table is
// what the reference compiles in today (c_lib/BG1_trained_ldpc_weights.c:25-33,
// BG2_trained_ldpc_weights.c): for 32 iterations, alpha by the row-degree
// rule (26623 for degree <= 4, 24575 for 5..8, 22527 above) and beta 0.
struct TrainedTable {
  std::vector<uint32_t> ab;
  int T = 0;
  uint64_t generation = 0;
};
TrainedTable g_trained[2];
uint64_t g_trained_gen = 1;

void default_trained(int bgn, TrainedTable* t) {
  const BaseGraph& g = base_graph(bgn);
  t->T = 32;
  t->ab.assign((size_t)t->T * g.rows, 0u);
  for (int it = 0; it < t->T; ++it) {
    for (int r = 0; r < g.rows; ++r) {
      const int d = g.degree[r];
      const int16_t a = d <= 4 ? 26623 : (d <= 8 ? 24575 : 22527);
      t->ab[(size_t)it * g.rows + r] = pack_ab(a, 0);
    }
  }
  t->generation = g_trained_gen++;
}

TrainedTable& trained(int bgn) {
  TrainedTable& t = g_trained[bgn == 1 ? 0 : 1];
  if (t.T == 0) default_trained(bgn, &t);
  return t;
}

struct Buffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

int ensure(Buffer* b, size_t bytes) {
  if (b->bytes >= bytes && b->ptr) return 0;
  if (b->ptr) cudaFree(b->ptr);
  b->ptr = nullptr;
  b->bytes = 0;
  size_t want = std::max(bytes, (size_t)256);
  cudaError_t e = cudaMalloc(&b->ptr, want);
  if (e != cudaSuccess) {
    b->ptr = nullptr;
    return (int)e;
  }
  b->bytes = want;
  return 0;
}

// Per-device state: CRC position tables, algo-2 tables, the soft buffer and
// staging buffers of the single-code-block ABI, and per-stream scratch.
struct DeviceState {
  bool init = false;
  uint32_t* crc_tab = nullptr;      // [4][kMaxB]
  Buffer trained_dev[2];
  uint64_t trained_gen[2] = {0, 0};
  // single-code-block ABI
  int16_t* harq = nullptr;          // [68*384] int16, process-wide soft buffer
  Buffer one_llr, one_bits, one_stat;
  Buffer one_info, one_rm;            // single-code-block encoder staging
  Buffer ch_in, ch_out;               // host-buffer channel staging
  std::map<cudaStream_t, Buffer> train_scratch;   // tape + carry of the training backward
  cudaStream_t one_stream = nullptr;
  // host-buffer batched API
  struct HostStage {
    Buffer llr, bits, stat, iters;
    cudaStream_t copy = nullptr;                   // copy-engine stream of the pipeline
    cudaStream_t comp[4] = {nullptr, nullptr, nullptr, nullptr};   // decode streams: chunks rotate over them
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> h2d, dec;             // per chunk
  };
  std::map<cudaStream_t, HostStage> host_stage;
  std::map<cudaStream_t, Buffer> scratch;
  std::map<cudaStream_t, Buffer> queue;   // fixed point: code-block queue head + finished-CTA count
  int num_sms = 0;
  // CTAs per SM by (kernel, clip variant, block, dynamic shared memory): the
  // driver query costs more than a small decode's host work, so it runs once
  std::map<uint64_t, int> occupancy;
  // pinned staging of the single-code-block ABI: LLRs in, status and hard bits out
  void* one_pin = nullptr;
  size_t one_pin_bytes = 0;
};

std::map<int, DeviceState> g_dev;

int device_state(DeviceState** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  DeviceState& st = g_dev[dev];
  if (!st.init) {
    e = cudaDeviceGetAttribute(&st.num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int)e;
    std::vector<uint32_t> tab((size_t)4 * kMaxB);
    for (int t = 0; t < 4; ++t) crc_position_table(t, tab.data() + (size_t)t * kMaxB);
    e = cudaMalloc(&st.crc_tab, tab.size() * sizeof(uint32_t));
    if (e != cudaSuccess) return (int)e;
    e = cudaMemcpy(st.crc_tab, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return (int)e;
    e = cudaMalloc(&st.harq, sizeof(int16_t) * kMaxCols * kMaxZc);
    if (e != cudaSuccess) return (int)e;
    e = cudaMemset(st.harq, 0, sizeof(int16_t) * kMaxCols * kMaxZc);
    if (e != cudaSuccess) return (int)e;
    e = cudaStreamCreateWithFlags(&st.one_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return (int)e;
    st.init = true;
  }
  *out = &st;
  return 0;
}

int trained_device_table(DeviceState* st, int bgn, const uint32_t** ptr, int* T) {
  TrainedTable& t = trained(bgn);
  const int k = bgn == 1 ? 0 : 1;
  if (st->trained_gen[k] != t.generation) {
    int e = ensure(&st->trained_dev[k], t.ab.size() * sizeof(uint32_t));
    if (e) return e;
    cudaError_t ce = cudaMemcpy(st->trained_dev[k].ptr, t.ab.data(), t.ab.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return (int)ce;
    st->trained_gen[k] = t.generation;
  }
  *ptr = static_cast<const uint32_t*>(st->trained_dev[k].ptr);
  *T = t.T;
  return 0;
}

struct Plan {
  DecodeParams p;
  int grid, block, smem;
  int clip;   // check-node arithmetic variant of the fixed-point kernel (fixed_clip_mode)
  int algo;
  size_t scratch_bytes;
};

// Fill the launch parameters of one uniform batch.
int make_plan(const CodeParams& cp, const ldpc_decoder_cfg_t& dc, int num_cw, DeviceState* st, Plan* plan) {
  DecodeParams& p = plan->p;
  memset(&p, 0, sizeof(p));
  const BaseGraph& g = base_graph(cp.bgn);
  p.Zc = cp.Zc;
  p.R = g.rows;
  p.lq_len = cp.lq_len;
  p.B = cp.B;
  p.K = cp.K;
  p.F = cp.F;
  p.N = cp.N;
  p.Nv = cp.Nv;
  p.E = cp.E;
  p.Qm = cp.Qm;
  p.symbols = cp.symbols;
  p.c0 = cp.c0;
  p.max_it = dc.max_iterations;
  p.harq_on = cp.harq_on;
  p.fill = dc.filling_bit_value;
  p.max_llr = dc.max_llr;
  p.min_llr = dc.min_llr;
  p.crc_tab = st->crc_tab + (size_t)cp.crctype * kMaxB;
  for (int e = 0; e < g.nnz; ++e) {
    const uint32_t colbase = (uint32_t)g.col[e] * (uint32_t)cp.Zc;
    const uint32_t sh = (uint32_t)(g.vij[cp.iLS][e] % cp.Zc);
    p.edge[e] = colbase | (sh << 16);
    p.edge_cs4[e] = make_uint2(4u * colbase, 4u * sh);
  }
  for (int r = 0; r <= g.rows; ++r) p.row_off[r] = g.row_off[r];

  const int algo = dc.algo;
  plan->algo = algo;
  const bool fixed = algo == 1 || algo == 2 || algo == 3;
  // Groups (lane pairs, or code blocks for the float kernels) per CTA: as many
  // as 384 threads hold, but for a small batch no more than spreading it over
  // all SMs needs, so a few blocks do not share one SM while others idle, and a
  // single block runs in a CTA as wide as Zc (its layer barriers wait for no
  // idle warps).
  {
    const int gmax = std::max(1, kThreadsTarget / cp.Zc);
    const int units = fixed ? (num_cw + 1) / 2 : num_cw;
    const int spread = (units + st->num_sms - 1) / std::max(st->num_sms, 1);
    p.G = std::max(1, std::min(gmax, spread));
  }
  p.nact = p.G * cp.Zc;
  plan->block = (p.nact + 31) & ~31;
  plan->smem = p.G * cp.lq_len * 4;
  p.num_cw = num_cw;
  if (fixed) {
    const int pairs = (num_cw + 1) / 2;
    p.num_items = (pairs + p.G - 1) / p.G;
  } else {
    p.num_items = (num_cw + p.G - 1) / p.G;
  }
  // Alpha/beta source.
  const int16_t alpha = (int16_t)dc.alpha;
  const int16_t beta = (int16_t)dc.beta;
  if (algo == 1) {
    for (int r = 0; r < g.rows; ++r) p.w_inline[r] = pack_ab(alpha, beta);
  } else if (algo == 3) {
    for (int r = 0; r < g.rows; ++r) p.w_inline[r] = pack_ab(degree_alpha(g.degree[r]), beta);
  } else if (algo == 2) {
    int e = trained_device_table(st, cp.bgn, &p.weights, &p.weights_T);
    if (e) return e;
  }
  p.rr_scatter = cp.E <= cp.Nv;
  p.qm_magic = qm_magic(cp.Qm);
  p.one = 1u;
  p.f_alpha = (float)dc.alpha / 32768.0f;
  p.f_beta = (float)dc.beta / 128.0f;
  p.f_max = (float)dc.max_llr / 128.0f;
  p.f_min = (float)dc.min_llr / 128.0f;
  plan->clip = fixed_clip_mode(dc, p.w_inline, g.rows);

  // Scratch layout per CTA, layer by layer.
  uint32_t off = 0;
  for (int r = 0; r < g.rows; ++r) {
    p.lr_off[r] = off;
    const int deg = g.degree[r];
    int planes;
    if (algo == 0) {
      planes = deg;
    } else if (fixed) {
      planes = fixed_row_planes(deg);
    } else {
      planes = 4;
    }
    // The fixed-point kernel addresses its planes with a compile-time stride.
    off += (uint32_t)planes * (uint32_t)(fixed ? kThreadsTarget : p.nact);
  }
  p.lr_off[g.rows] = off;
  p.scratch_words = off;

  const uint64_t key = ((uint64_t)(fixed ? 1 : algo == 4 ? 2 : 3) << 56) | ((uint64_t)(fixed ? plan->clip : 0) << 48) |
                       ((uint64_t)plan->block << 32) | (uint64_t)(uint32_t)plan->smem;
  int occ;
  auto hit = st->occupancy.find(key);
  if (hit != st->occupancy.end()) {
    occ = hit->second;
  } else {
    if (fixed) {
      occ = occupancy_fixed(plan->block, plan->smem, plan->clip, true);
    } else if (algo == 4) {
      occ = occupancy_float_minsum(plan->block, plan->smem);
    } else {
      occ = occupancy_float_bp(plan->block, plan->smem);
    }
    st->occupancy[key] = occ;
  }
  if (occ < 1) occ = 1;
  plan->grid = std::min(p.num_items, occ * st->num_sms);
  if (plan->grid < 1) plan->grid = 1;
  plan->scratch_bytes = (size_t)plan->grid * (size_t)p.scratch_words * sizeof(uint32_t);
  return 0;
}

int launch_plan(Plan* plan, void* stream) {
  switch (plan->algo) {
    case 1:
    case 2:
    case 3:
      return launch_fixed(plan->p, plan->grid, plan->block, plan->smem, plan->clip, stream);
    case 4:
      return launch_float_minsum(plan->p, plan->grid, plan->block, plan->smem, stream);
    default:
      return launch_float_bp(plan->p, plan->grid, plan->block, plan->smem, stream);
  }
}

int scratch_for(DeviceState* st, cudaStream_t s, size_t bytes, uint32_t** out) {
  Buffer& b = st->scratch[s];
  int e = ensure(&b, bytes);
  if (e) return e;
  *out = static_cast<uint32_t*>(b.ptr);
  return 0;
}

// Shared body of the batched entry points.  `lock` must be held.
int32_t decode_batch_locked(const int16_t* d_llr, int64_t llr_stride, int32_t num_cw,
                            const ldpc_in_config_t* in, const ldpc_decoder_cfg_t* dc, uint8_t* d_bits,
                            int64_t bits_stride, int32_t* d_status, int32_t* d_iters, void* d_app,
                            int64_t app_stride, int16_t* d_harq, int64_t harq_stride, void* stream) {
  if (!in || !dc || num_cw < 0) return NRLDPC_ERR_ARG;
  CodeParams cp;
  if (derive_params(*in, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  if (dc->algo > 4) {
    fprintf(stderr, "nrldpc: invalid decoding algorithm selection: %u\n", dc->algo);
    return NRLDPC_ERR_ALGO;
  }
  if (num_cw == 0) return NRLDPC_OK;
  if (!d_llr || llr_stride < cp.E) return NRLDPC_ERR_ARG;
  if (d_bits && bits_stride < (cp.B + 7) / 8) return NRLDPC_ERR_ARG;
  if (d_app && app_stride < cp.lq_len) return NRLDPC_ERR_ARG;
  if (d_harq && harq_stride < cp.lq_len) return NRLDPC_ERR_ARG;
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  Plan plan;
  if (make_plan(cp, *dc, num_cw, st, &plan) != 0) return NRLDPC_ERR_CUDA;
  uint32_t* scratch = nullptr;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (scratch_for(st, s, plan.scratch_bytes, &scratch) != 0) return NRLDPC_ERR_CUDA;
  DecodeParams& p = plan.p;
  if (p.num_items > plan.grid) {
    // More than one wave: work comes from the stream's queue (zeroed once,
    // rewound by each launch's last CTA): fixed point refills half lanes from
    // it, the float kernels take work items from it.  Within one wave there is
    // nothing to balance, and the fixed work items are a little faster.
    Buffer& q = st->queue[s];
    if (!q.ptr && (ensure(&q, 256) != 0 || cudaMemsetAsync(q.ptr, 0, 256, s) != cudaSuccess))
      return NRLDPC_ERR_CUDA;
    p.cursor = static_cast<int32_t*>(q.ptr);
  }
  p.llr = d_llr;
  p.llr_stride = llr_stride;
  p.rr_vec = (reinterpret_cast<uintptr_t>(d_llr) % 16 == 0) && (llr_stride % 8 == 0);
  p.bits = d_bits;
  p.bits_stride = bits_stride;
  p.status = d_status;
  p.iters = d_iters;
  p.app = d_app;
  p.app_stride = app_stride;
  p.harq = d_harq;
  p.harq_stride = harq_stride;
  p.scratch = scratch;
  if (launch_plan(&plan, stream) != 0) return NRLDPC_ERR_CUDA;
  return NRLDPC_OK;
}

// One code block from host memory, through the process-wide soft buffer.
int32_t decode_one(int16_t* LLr, uint8_t* hardbits, ldpc_in_config_t* inconfig, ldpc_decoder_cfg_t* dcfg) {
  if (!inconfig || !dcfg) return NRLDPC_ERR_CONFIG;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  if (cp.E > 0 && !LLr) return NRLDPC_ERR_CUDA;
  const int nbytes = (cp.B + 7) / 8;
  if (ensure(&st->one_llr, sizeof(int16_t) * std::max(cp.E, 1)) || ensure(&st->one_bits, (size_t)nbytes) ||
      ensure(&st->one_stat, 2 * sizeof(int32_t)))
    return NRLDPC_ERR_CUDA;
  // Pinned staging [status (16 B) | hard bits | LLRs]: copies from and to the
  // caller's pageable buffers go through it, so the device copies are plain
  // asynchronous transfers.
  const size_t bits_off = 16, llr_off = bits_off + (((size_t)nbytes + 15) & ~(size_t)15);
  const size_t pin_bytes = llr_off + sizeof(int16_t) * (size_t)std::max(cp.E, 1);
  if (st->one_pin_bytes < pin_bytes) {
    if (st->one_pin) cudaFreeHost(st->one_pin);
    st->one_pin = nullptr;
    st->one_pin_bytes = 0;
    const size_t want = std::max(pin_bytes, (size_t)(16 + 1056 + 2 * 26112));   // up to BG1 Zc=384 at E = N
    if (cudaHostAlloc(&st->one_pin, want, cudaHostAllocDefault) != cudaSuccess) {
      st->one_pin = nullptr;
      return NRLDPC_ERR_CUDA;
    }
    st->one_pin_bytes = want;
  }
  char* pin = static_cast<char*>(st->one_pin);
  cudaStream_t s = st->one_stream;
  if (cp.E > 0) {
    memcpy(pin + llr_off, LLr, sizeof(int16_t) * cp.E);
    if (cudaMemcpyAsync(st->one_llr.ptr, pin + llr_off, sizeof(int16_t) * cp.E, cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
      return NRLDPC_ERR_CUDA;
  }
  // The reference recovers into its soft buffer before it looks at algo
  // (c_lib/c_ldpc_5g_decoder.c:44-78), so an invalid algo still updates the
  // buffer: run the recovery alone (zero iterations) in that case.
  ldpc_decoder_cfg_t run = *dcfg;
  const bool bad_algo = dcfg->algo > 4;
  if (bad_algo) {
    run.algo = 1;
    run.max_iterations = 0;
  }
  int32_t* d_stat = static_cast<int32_t*>(st->one_stat.ptr);
  int32_t rc = decode_batch_locked(static_cast<int16_t*>(st->one_llr.ptr), std::max(cp.E, 1), 1, inconfig,
                                   &run, static_cast<uint8_t*>(st->one_bits.ptr), nbytes, d_stat, nullptr,
                                   nullptr, 0, st->harq, kMaxCols * kMaxZc, s);
  if (rc != NRLDPC_OK) return rc;
  if (cudaMemcpyAsync(pin, d_stat, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return NRLDPC_ERR_CUDA;
  // With zero iterations the reference leaves the caller's bits untouched.
  const bool copy_bits = run.max_iterations > 0 && hardbits;
  if (copy_bits && cudaMemcpyAsync(pin + bits_off, st->one_bits.ptr, nbytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return NRLDPC_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return NRLDPC_ERR_CUDA;
  int32_t status = 1;
  memcpy(&status, pin, sizeof(int32_t));
  if (copy_bits) memcpy(hardbits, pin + bits_off, nbytes);
  if (bad_algo) {
    fprintf(stderr, "nrldpc: invalid decoding algorithm selection: %u\n", dcfg->algo);
    return NRLDPC_ERR_ALGO;
  }
  return status;
}

// Launch parameters of the batched encoder for one configuration.
void make_encode_params(const CodeParams& cp, DeviceState* st, EncodeParams* e) {
  memset(e, 0, sizeof(*e));
  const BaseGraph& g = base_graph(cp.bgn);
  e->bgn = cp.bgn;
  e->Zc = cp.Zc;
  e->R = g.rows;
  e->cols = g.cols;
  e->A = cp.A;
  e->B = cp.B;
  e->K = cp.K;
  e->F = cp.F;
  e->N = cp.N;
  e->Nv = cp.Nv;
  e->E = cp.E;
  e->Qm = cp.Qm;
  e->symbols = cp.symbols;
  e->c0 = cp.c0;
  e->Kb = cp.K / cp.Zc;
  for (int i = 0; i < g.nnz; ++i) e->edge[i] = (uint32_t)g.col[i] | ((uint32_t)(g.vij[cp.iLS][i] % cp.Zc) << 16);
  for (int r = 0; r <= g.rows; ++r) e->row_off[r] = g.row_off[r];
  // Core parity circulants (c_lib/ldpc_encoder.c:95-109): BG1 row 0 / row 1 at
  // base column 22, BG2 row 0 / row 2 at base column 10.
  if (cp.bgn == 1) {
    e->shift0 = g.vij[cp.iLS][g.row_off[0] + 17] % cp.Zc;
    e->shift1 = g.vij[cp.iLS][g.row_off[1] + 16] % cp.Zc;
  } else {
    e->shift0 = g.vij[cp.iLS][g.row_off[0] + 6] % cp.Zc;
    e->shift1 = g.vij[cp.iLS][g.row_off[2] + 5] % cp.Zc;
  }
  e->crc_tab = st->crc_tab + (size_t)cp.crctype * kMaxB;
}

int32_t encode_one(uint8_t* infobytes, uint8_t* rm_bytes, ldpc_in_config_t* inconfig) {
  if (!inconfig) return NRLDPC_ERR_CONFIG;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  const int in_bytes = std::max(cp.A / 8, 1), out_bytes = std::max((cp.E + 7) / 8, 1);
  if ((cp.A > 0 && !infobytes) || (cp.E > 0 && !rm_bytes)) return NRLDPC_ERR_CUDA;
  if (ensure(&st->one_info, (size_t)in_bytes) || ensure(&st->one_rm, (size_t)out_bytes)) return NRLDPC_ERR_CUDA;
  cudaStream_t s = st->one_stream;
  if (cp.A > 0 && cudaMemcpyAsync(st->one_info.ptr, infobytes, cp.A / 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return NRLDPC_ERR_CUDA;
  EncodeParams e;
  make_encode_params(cp, st, &e);
  e.num_cw = 1;
  e.info = static_cast<const uint8_t*>(st->one_info.ptr);
  e.info_stride = in_bytes;
  e.rm = static_cast<uint8_t*>(st->one_rm.ptr);
  e.rm_stride = out_bytes;
  if (launch_encode(e, s) != 0) return NRLDPC_ERR_CUDA;
  if (cp.E > 0 && cudaMemcpyAsync(rm_bytes, st->one_rm.ptr, (cp.E + 7) / 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return NRLDPC_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return NRLDPC_ERR_CUDA;
  return NRLDPC_OK;
}

// Launch geometry of the training kernels for one configuration.  One code
// block needs at least one (N+2Zc)-value array of shared memory (the backward
// can hold LQ and dLQ in the same array at different times); the float64
// variant runs fewer blocks per CTA.
int make_train_params(const ldpc_in_config_t* cfg, int32_t T, int32_t batch, double clip, bool f64, TrainParams* p,
                      int* block, int* smem_fwd, int* smem_bwd) {
  CodeParams cp;
  if (!cfg || derive_params(*cfg, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  if (T < 1 || batch < 0) return NRLDPC_ERR_ARG;
  memset(p, 0, sizeof(*p));
  const BaseGraph& g = base_graph(cp.bgn);
  const int real = f64 ? 8 : 4;
  const int smem_cap = 227 * 1024 - 1024;   // opt-in shared memory per block, less the static reduction buffer
  int G = std::max(1, kThreadsTarget / cp.Zc);
  while (G > 1 && G * cp.lq_len * real > smem_cap) --G;
  if (G * cp.lq_len * real > smem_cap) return NRLDPC_ERR_CONFIG;
  p->Zc = cp.Zc;
  p->R = g.rows;
  p->n = cp.lq_len;
  p->G = G;
  p->nnz = g.nnz;
  p->T = T;
  p->batch = batch;
  p->msg_words = (f64 ? 6 : 4) * cp.Zc;
  p->clip = clip > 0.0 ? clip : INFINITY;
  for (int e = 0; e < g.nnz; ++e)
    p->edge[e] = (uint32_t)g.col[e] * (uint32_t)cp.Zc | ((uint32_t)(g.vij[cp.iLS][e] % cp.Zc) << 16);
  for (int r = 0; r <= g.rows; ++r) p->row_off[r] = g.row_off[r];
  *block = (p->G * cp.Zc + 31) & ~31;
  *smem_fwd = p->G * cp.lq_len * real;
  *smem_bwd = p->G * cp.lq_len * real;   // with LQ and dLQ sharing the array; pick_train_groups decides
  return NRLDPC_OK;
}

// Code blocks per CTA (G) that put the most code blocks on an SM, given the
// kernel's registers and shared memory (one (N+2Zc)-value array per block in
// the forward; two in the backward, or one when LQ and dLQ share it, which the
// backward does only where that puts more blocks on an SM, since it costs a
// round trip of dLQ through global memory per iteration); the largest G among
// equals.  Returns the blocks per SM of that choice and sets p->G, p->alias,
// *block, *smem.
int pick_train_groups(TrainParams* p, bool backward, bool f64, int* block, int* smem) {
  const int real = f64 ? 8 : 4;
  const int smem_cap = 227 * 1024 - 1024;
  const int gmax = std::max(1, kThreadsTarget / p->Zc);
  int best_g = 0, best_cw = 0, best_occ = 0, best_alias = 0;
  for (int alias = 0; alias <= (backward ? 1 : 0); ++alias) {
    const int per = (backward && !alias ? 2 : 1) * p->n * real;
    for (int G = gmax; G >= 1; --G) {
      if (G * per > smem_cap) continue;
      const int blk = (G * p->Zc + 31) & ~31;
      const int occ = occupancy_train(backward, f64, p->R == 42, blk, G * per, alias != 0);
      if (occ * G > best_cw) {
        best_cw = occ * G;
        best_g = G;
        best_occ = occ;
        best_alias = alias;
      }
    }
  }
  if (best_g == 0) return 0;
  p->G = best_g;
  p->alias = best_alias;
  *block = (best_g * p->Zc + 31) & ~31;
  *smem = best_g * (backward && !best_alias ? 2 : 1) * p->n * real;
  return best_occ;
}

int train_forward(const void* d_llr, int32_t batch, const ldpc_in_config_t* cfg, int32_t iterations,
                  const void* d_alpha, const void* d_beta, double clip, void* d_final, void* d_iter, void* d_ck_lq,
                  uint32_t* d_ck_lr, void* stream, bool f64) {
  TrainParams p;
  int block, smem_f, smem_b;
  const int rc = make_train_params(cfg, iterations, batch, clip, f64, &p, &block, &smem_f, &smem_b);
  if (rc != NRLDPC_OK) return rc;
  if (batch == 0) return NRLDPC_OK;
  if (!d_llr || !d_alpha || !d_beta || !d_final || !d_ck_lq || !d_ck_lr) return NRLDPC_ERR_ARG;
  p.llr = d_llr;
  p.alpha = d_alpha;
  p.beta = d_beta;
  p.final_llr = d_final;
  p.iter_llr = d_iter;
  p.ck_lq = d_ck_lq;
  p.ck_lr = d_ck_lr;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int occ = std::max(1, pick_train_groups(&p, false, f64, &block, &smem_f));
  const int items = (batch + p.G - 1) / p.G;
  const int grid = std::max(1, std::min(items, occ * sms));
  return launch_train_forward(p, f64, grid, block, smem_f, stream) == 0 ? NRLDPC_OK : NRLDPC_ERR_CUDA;
}

int train_backward(const void* d_llr, int32_t batch, const ldpc_in_config_t* cfg, int32_t iterations,
                   const void* d_alpha, const void* d_beta, double clip, int32_t detach, const void* d_ck_lq,
                   const uint32_t* d_ck_lr, const void* d_g_final, const void* d_g_iter, void* d_g_llr,
                   void* d_g_alpha, void* d_g_beta, void* stream, bool f64) {
  TrainParams p;
  int block, smem_f, smem_b;
  const int rc = make_train_params(cfg, iterations, batch, clip, f64, &p, &block, &smem_f, &smem_b);
  if (rc != NRLDPC_OK) return rc;
  if (batch == 0) return NRLDPC_OK;
  if (!d_llr || !d_alpha || !d_beta || !d_ck_lq || !d_ck_lr || !d_g_llr || !d_g_alpha || !d_g_beta)
    return NRLDPC_ERR_ARG;
  p.llr = d_llr;
  p.alpha = d_alpha;
  p.beta = d_beta;
  p.detach = detach ? 1 : 0;
  p.ck_lq = const_cast<void*>(d_ck_lq);
  p.ck_lr = const_cast<uint32_t*>(d_ck_lr);
  p.g_final = d_g_final;
  p.g_iter = d_g_iter;
  p.g_llr = d_g_llr;
  p.g_alpha = d_g_alpha;
  p.g_beta = d_g_beta;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  const int occ = std::max(1, pick_train_groups(&p, true, f64, &block, &smem_b));
  const int items = (batch + p.G - 1) / p.G;
  const int grid = std::max(1, std::min(items, occ * st->num_sms));
  p.scratch_per_cta = (int64_t)p.G * p.nnz * p.Zc;
  const size_t real = f64 ? 8 : 4;
  Buffer& b = st->train_scratch[reinterpret_cast<cudaStream_t>(stream)];
  if (ensure(&b, 2 * real * (size_t)grid * (size_t)p.scratch_per_cta)) return NRLDPC_ERR_CUDA;
  p.tape = b.ptr;
  p.carry = static_cast<char*>(b.ptr) + real * (size_t)grid * (size_t)p.scratch_per_cta;
  return launch_train_backward(p, f64, grid, block, smem_b, stream) == 0 ? NRLDPC_OK : NRLDPC_ERR_CUDA;
}

}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Device tables of the current device, for other translation units.
int device_crc_table(const uint32_t** tab) {
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  *tab = st->crc_tab;
  return NRLDPC_OK;
}

int device_trained_table(int bgn, const uint32_t** ptr, int* T) {
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  return trained_device_table(st, bgn, ptr, T) == 0 ? NRLDPC_OK : NRLDPC_ERR_CUDA;
}

// Read-only views of the algo-2 / algo-3 tables for other translation units.
int16_t current_degree_alpha(int deg) {
  std::lock_guard<std::mutex> lock(g_mu);
  return degree_alpha(deg);
}

uint64_t current_trained_table(int bgn, std::vector<uint32_t>* ab, int* T) {
  std::lock_guard<std::mutex> lock(g_mu);
  TrainedTable& t = trained(bgn);
  *ab = t.ab;
  *T = t.T;
  return t.generation;
}

}  // namespace nrldpc

using namespace nrldpc;

extern "C" {

int gen_ldpc_parameters(ldpc_config_t* params, ldpc_in_config_t* inconfig) {
  if (!params || !inconfig) return -1;
  params->bgn = inconfig->bgn;
  params->A = inconfig->A;
  params->crctype = inconfig->crctype;
  params->E = inconfig->E;
  params->rv = inconfig->rv;
  params->Qm = inconfig->Qm;
  params->HARQ_on = inconfig->HARQ_on;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return -1;
  params->B = (uint16_t)cp.B;
  params->Zc = (uint16_t)cp.Zc;
  params->iLS = (uint16_t)cp.iLS;
  params->K = (uint16_t)cp.K;
  params->F = (uint16_t)cp.F;
  params->N = (uint16_t)cp.N;
  params->k0 = (uint16_t)cp.k0;
  BaseGraph& g = const_cast<BaseGraph&>(base_graph(cp.bgn));
  params->Vij_array = g.vij[cp.iLS];
  params->HBG_array = g.col;
  params->HBG_offset_array = g.row_off;
  return 0;
}

uint32_t calculate_crc(const uint8_t* data, int len, int crctype) { return crc_remainder(data, len, crctype); }

int32_t cuda_ldpc_5g_decode(int16_t* LLr, uint8_t* hardbits, ldpc_in_config_t* inconfig,
                            ldpc_decoder_cfg_t* decoder_config) {
  return decode_one(LLr, hardbits, inconfig, decoder_config);
}

int32_t c_ldpc_5g_decode(int16_t* LLr, uint8_t* hardbits, ldpc_in_config_t* inconfig,
                         ldpc_decoder_cfg_t* decoder_config) {
  return decode_one(LLr, hardbits, inconfig, decoder_config);
}

int32_t nrldpc_decode_batch(const int16_t* d_llr, int64_t llr_stride, int32_t num_cw,
                            const ldpc_in_config_t* inconfig, const ldpc_decoder_cfg_t* decoder_cfg,
                            uint8_t* d_hardbits, int64_t bits_stride, int32_t* d_status, int32_t* d_iterations,
                            void* d_app, int64_t app_stride, int16_t* d_harq, int64_t harq_stride,
                            void* stream) {
  std::lock_guard<std::mutex> lock(g_mu);
  return decode_batch_locked(d_llr, llr_stride, num_cw, inconfig, decoder_cfg, d_hardbits, bits_stride, d_status,
                             d_iterations, d_app, app_stride, d_harq, harq_stride, stream);
}

int32_t nrldpc_decode_batch_host(const int16_t* h_llr, int64_t llr_stride, int32_t num_cw,
                                 const ldpc_in_config_t* inconfig, const ldpc_decoder_cfg_t* decoder_cfg,
                                 uint8_t* h_hardbits, int64_t bits_stride, int32_t* h_status,
                                 int32_t* h_iterations, void* stream) {
  if (!inconfig || !decoder_cfg || num_cw < 0) return NRLDPC_ERR_ARG;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  if (decoder_cfg->algo > 4) return NRLDPC_ERR_ALGO;
  if (num_cw == 0) return NRLDPC_OK;
  if (!h_llr || llr_stride < cp.E || !h_hardbits) return NRLDPC_ERR_ARG;
  const int nbytes = (cp.B + 7) / 8;
  if (bits_stride < nbytes) return NRLDPC_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  DeviceState::HostStage& hs = st->host_stage[s];
  const size_t llr_bytes = sizeof(int16_t) * (size_t)num_cw * (size_t)llr_stride;
  const size_t bit_bytes = (size_t)num_cw * (size_t)bits_stride;
  if (ensure(&hs.llr, llr_bytes) || ensure(&hs.bits, bit_bytes) || ensure(&hs.stat, sizeof(int32_t) * num_cw) ||
      ensure(&hs.iters, sizeof(int32_t) * num_cw))
    return NRLDPC_ERR_CUDA;
  if (!hs.copy) {
    if (cudaStreamCreateWithFlags(&hs.copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&hs.comp[0], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&hs.comp[1], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&hs.comp[2], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&hs.comp[3], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&hs.start, cudaEventDisableTiming) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
  }
  // Chunks: chunk k+1's host-to-device copy overlaps the decode of the chunks
  // before it.  The first three are a quarter, a quarter and half a kernel
  // wave, the rest whole waves (at most 32 chunks): the first copy, the only
  // one nothing hides, is small, and decoding starts while the next chunks
  // arrive.  Chunks rotate over four decode streams, so the small first chunks
  // run side by side and every chunk's CTAs start on the SMs that earlier
  // chunks' finishers leave free (no tail per chunk).
  Plan probe;
  if (make_plan(cp, *decoder_cfg, num_cw, st, &probe) != 0) return NRLDPC_ERR_CUDA;
  const bool fixed = decoder_cfg->algo >= 1 && decoder_cfg->algo <= 3;
  const int64_t wave_cw = (int64_t)(fixed ? 2 : 1) * probe.p.G * probe.grid;
  std::vector<int64_t> cuts{0};   // chunk k covers blocks [cuts[k], cuts[k+1])
  constexpr int kMaxChunks = 32;
  if (wave_cw >= 8 && num_cw >= 3 * wave_cw) {
    const int64_t q = (wave_cw / 4 + 1) & ~(int64_t)1;   // even: whole lane pairs
    const int64_t want = (num_cw + kMaxChunks - 4) / (kMaxChunks - 3);
    const int64_t body = std::max<int64_t>(wave_cw, (want + wave_cw - 1) / wave_cw * wave_cw);
    for (const int64_t c : {q, q, 2 * q}) cuts.push_back(cuts.back() + c);
    while (cuts.back() < num_cw) cuts.push_back(std::min<int64_t>(num_cw, cuts.back() + body));
  } else {
    cuts.push_back(num_cw);
  }
  const int nchunks = (int)cuts.size() - 1;
  while ((int)hs.h2d.size() < nchunks) {
    cudaEvent_t a, b;
    if (cudaEventCreateWithFlags(&a, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b, cudaEventDisableTiming) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    hs.h2d.push_back(a);
    hs.dec.push_back(b);
  }
  // work already queued on the caller's stream comes first
  if (cudaEventRecord(hs.start, s) != cudaSuccess || cudaStreamWaitEvent(hs.copy, hs.start, 0) != cudaSuccess ||
      cudaStreamWaitEvent(hs.comp[0], hs.start, 0) != cudaSuccess ||
      cudaStreamWaitEvent(hs.comp[1], hs.start, 0) != cudaSuccess ||
      cudaStreamWaitEvent(hs.comp[2], hs.start, 0) != cudaSuccess ||
      cudaStreamWaitEvent(hs.comp[3], hs.start, 0) != cudaSuccess)
    return NRLDPC_ERR_CUDA;
  int16_t* d_llr = static_cast<int16_t*>(hs.llr.ptr);
  uint8_t* d_bits = static_cast<uint8_t*>(hs.bits.ptr);
  int32_t* d_stat = static_cast<int32_t*>(hs.stat.ptr);
  int32_t* d_iters = static_cast<int32_t*>(hs.iters.ptr);
  for (int k = 0; k < nchunks; ++k) {
    const int64_t c0 = cuts[k], n = cuts[k + 1] - cuts[k];
    const size_t off = (size_t)c0 * (size_t)llr_stride;
    if (cudaMemcpyAsync(d_llr + off, h_llr + off, sizeof(int16_t) * (size_t)n * (size_t)llr_stride,
                        cudaMemcpyHostToDevice, hs.copy) != cudaSuccess ||
        cudaEventRecord(hs.h2d[k], hs.copy) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
  }
  for (int k = 0; k < nchunks; ++k) {
    const int64_t c0 = cuts[k], n = cuts[k + 1] - cuts[k];
    cudaStream_t comp = hs.comp[k & 3];
    if (cudaStreamWaitEvent(comp, hs.h2d[k], 0) != cudaSuccess) return NRLDPC_ERR_CUDA;
    const int32_t rc = decode_batch_locked(d_llr + (size_t)c0 * (size_t)llr_stride, llr_stride, (int32_t)n, inconfig,
                                           decoder_cfg, d_bits + (size_t)c0 * (size_t)bits_stride, bits_stride,
                                           d_stat + c0, d_iters + c0, nullptr, 0, nullptr, 0, comp);
    if (rc != NRLDPC_OK) return rc;
    if (cudaEventRecord(hs.dec[k], comp) != cudaSuccess || cudaStreamWaitEvent(hs.copy, hs.dec[k], 0) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    if (decoder_cfg->max_iterations > 0 &&
        cudaMemcpyAsync(h_hardbits + (size_t)c0 * (size_t)bits_stride, d_bits + (size_t)c0 * (size_t)bits_stride,
                        (size_t)n * (size_t)bits_stride, cudaMemcpyDeviceToHost, hs.copy) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    if (h_status && cudaMemcpyAsync(h_status + c0, d_stat + c0, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost,
                                    hs.copy) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    if (h_iterations && cudaMemcpyAsync(h_iterations + c0, d_iters + c0, sizeof(int32_t) * (size_t)n,
                                        cudaMemcpyDeviceToHost, hs.copy) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
  }
  if (cudaStreamSynchronize(hs.copy) != cudaSuccess) return NRLDPC_ERR_CUDA;
  return NRLDPC_OK;
}

int32_t nrldpc_set_trained_weights(uint16_t bgn, const int16_t* alpha, const int16_t* beta,
                                   int32_t num_iterations) {
  if (bgn != 1 && bgn != 2) return NRLDPC_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  TrainedTable& t = g_trained[bgn == 1 ? 0 : 1];
  if (!alpha) {
    default_trained(bgn, &t);
    return NRLDPC_OK;
  }
  if (num_iterations < 1 || num_iterations > 65535) return NRLDPC_ERR_ARG;
  const BaseGraph& g = base_graph(bgn);
  t.T = num_iterations;
  t.ab.assign((size_t)num_iterations * g.rows, 0u);
  for (size_t i = 0; i < t.ab.size(); ++i) t.ab[i] = pack_ab(alpha[i], beta ? beta[i] : (int16_t)0);
  t.generation = g_trained_gen++;
  return NRLDPC_OK;
}

int32_t nrldpc_set_degree_alpha(const int16_t* degree_alpha_values) {
  std::lock_guard<std::mutex> lock(g_mu);
  memcpy(g_degree_alpha, degree_alpha_values ? degree_alpha_values : kDefaultDegreeAlpha, sizeof(g_degree_alpha));
  g_degree_alpha_init = true;
  return NRLDPC_OK;
}

int64_t nrldpc_kernel_launch_count(void) { return g_launches.load(); }

const char* nrldpc_version(void) {
  return kBoundsChecked ? "nrldpc-b200 0.1.0 (sm_100a, bounds-checked debug build)" : "nrldpc-b200 0.1.0 (sm_100a)";
}

int32_t nrldpc_bounds_check_status(uint32_t* out, int32_t reset) {
  if (!out) return NRLDPC_ERR_ARG;
  out[0] = out[1] = out[2] = out[3] = 0u;
  if (!kBoundsChecked) return 0;
  // first record among the kernels' translation units (fixed-point, float, mixed)
  int (*readers[3])(uint32_t*, bool) = {bounds_read_fixed, bounds_read_float, bounds_read_mixed};
  for (auto rd : readers) {
    uint32_t r[4];
    if (rd(r, reset != 0) != 0) return NRLDPC_ERR_CUDA;
    if (out[0] == 0u && r[0] != 0u) memcpy(out, r, sizeof(r));
  }
  return 1;
}

int32_t nrldpc_encode_batch(const uint8_t* d_info, int64_t info_stride, int32_t num_cw,
                            const ldpc_in_config_t* inconfig, uint8_t* d_rm, int64_t rm_stride, void* stream) {
  if (!inconfig || num_cw < 0) return NRLDPC_ERR_ARG;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  if (num_cw == 0) return NRLDPC_OK;
  if (!d_info || !d_rm || info_stride < cp.A / 8 || rm_stride < (cp.E + 7) / 8) return NRLDPC_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  EncodeParams e;
  make_encode_params(cp, st, &e);
  e.num_cw = num_cw;
  e.info = d_info;
  e.info_stride = info_stride;
  e.rm = d_rm;
  e.rm_stride = rm_stride;
  return launch_encode(e, stream) == 0 ? NRLDPC_OK : NRLDPC_ERR_CUDA;
}

int32_t nrldpc_encode_batch_ncb(const uint8_t* d_info, int64_t info_stride, int32_t num_cw,
                                const ldpc_in_config_t* inconfig, int32_t ncb, uint8_t* d_rm, int64_t rm_stride,
                                void* stream) {
  if (!inconfig || num_cw < 0) return NRLDPC_ERR_ARG;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  if (ncb > 0 && ncb < cp.N) {
    if (ncb < cp.K - 2 * cp.Zc) return NRLDPC_ERR_CONFIG;
    // TS 38.212 Table 5.4.2.1-2 with Ncb < N
    static const int fa[4] = {0, 17, 33, 56}, fb[4] = {0, 13, 25, 43};
    const int f = (cp.bgn == 1 ? fa : fb)[cp.rv];
    cp.k0 = (int)(((int64_t)f * ncb) / ((int64_t)(cp.bgn == 1 ? 66 : 50) * cp.Zc)) * cp.Zc;
    cp.Nv = ncb - cp.F;
    const int fill_lo = cp.B - 2 * cp.Zc, fill_hi = cp.K - 2 * cp.Zc;
    cp.c0 = cp.k0 < fill_lo ? cp.k0 : (cp.k0 < fill_hi ? fill_lo : cp.k0 - cp.F);
  }
  if (num_cw == 0) return NRLDPC_OK;
  if (!d_info || !d_rm || info_stride < cp.A / 8 || rm_stride < (cp.E + 7) / 8) return NRLDPC_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return NRLDPC_ERR_CUDA;
  EncodeParams e;
  make_encode_params(cp, st, &e);
  e.num_cw = num_cw;
  e.info = d_info;
  e.info_stride = info_stride;
  e.rm = d_rm;
  e.rm_stride = rm_stride;
  return launch_encode(e, stream) == 0 ? NRLDPC_OK : NRLDPC_ERR_CUDA;
}

int32_t cuda_ldpc_5g_encode(uint8_t* infobytes, uint8_t* rm_bytes, ldpc_in_config_t* inconfig) {
  return encode_one(infobytes, rm_bytes, inconfig);
}

int32_t c_ldpc_5g_encode(uint8_t* infobytes, uint8_t* rm_bytes, ldpc_in_config_t* inconfig) {
  return encode_one(infobytes, rm_bytes, inconfig);
}

int32_t nrldpc_channel_batch(const uint8_t* d_rm, int64_t rm_stride, int32_t num_cw, int32_t E, int32_t Qm,
                             float noise_power_db, uint64_t seed, int16_t* d_llr, int64_t llr_stride,
                             float* d_symbols, void* stream) {
  float nv, sigma, A;
  if (num_cw < 0 || E < 0 || !channel_constants(Qm, noise_power_db, &nv, &sigma, &A) || E % Qm) return NRLDPC_ERR_ARG;
  if (num_cw == 0 || E == 0) return NRLDPC_OK;
  if (!d_rm || !d_llr || rm_stride < (E + 7) / 8 || llr_stride < E) return NRLDPC_ERR_ARG;
  return launch_channel(d_rm, rm_stride, num_cw, E, Qm, nv, sigma, A, seed, d_llr, llr_stride, d_symbols, stream) == 0
             ? NRLDPC_OK
             : NRLDPC_ERR_CUDA;
}

void nrldpc_channel_seed(uint64_t seed) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_channel_seed = seed;
  g_channel_calls = 0;
}

int tx_rx_process(const uint8_t* inbytes, size_t num_bits, uint16_t Qm, float noise_power_db, int16_t* llr_out) {
  float nv, sigma, A;
  if (!inbytes || !llr_out || num_bits == 0) return -1;
  if (!channel_constants(Qm, noise_power_db, &nv, &sigma, &A) || num_bits % Qm) return -1;
  if (num_bits > (size_t)INT32_MAX) return -1;
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState* st = nullptr;
  if (device_state(&st) != 0) return -1;
  const size_t in_bytes = (num_bits + 7) / 8;
  if (ensure(&st->ch_in, in_bytes) || ensure(&st->ch_out, num_bits * sizeof(int16_t))) return -1;
  cudaStream_t s = st->one_stream;
  const uint64_t seed = g_channel_seed ^ (0x9E3779B97F4A7C15ull * ++g_channel_calls);
  if (cudaMemcpyAsync(st->ch_in.ptr, inbytes, in_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return -1;
  if (launch_channel(static_cast<uint8_t*>(st->ch_in.ptr), (int64_t)in_bytes, 1, (int32_t)num_bits, Qm, nv, sigma, A,
                     seed, static_cast<int16_t*>(st->ch_out.ptr), (int64_t)num_bits, nullptr, s) != 0)
    return -1;
  if (cudaMemcpyAsync(llr_out, st->ch_out.ptr, num_bits * sizeof(int16_t), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return -1;
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
}

int32_t nrldpc_train_forward(const float* d_llr, int32_t batch, const ldpc_in_config_t* cfg, int32_t iterations,
                             const float* d_alpha, const float* d_beta, float clip, float* d_final, float* d_iter,
                             float* d_ck_lq, uint32_t* d_ck_lr, void* stream) {
  return train_forward(d_llr, batch, cfg, iterations, d_alpha, d_beta, clip, d_final, d_iter, d_ck_lq, d_ck_lr, stream,
                       false);
}

int32_t nrldpc_train_backward(const float* d_llr, int32_t batch, const ldpc_in_config_t* cfg, int32_t iterations,
                              const float* d_alpha, const float* d_beta, float clip, int32_t detach,
                              const float* d_ck_lq, const uint32_t* d_ck_lr, const float* d_g_final,
                              const float* d_g_iter, float* d_g_llr, float* d_g_alpha, float* d_g_beta,
                              void* stream) {
  return train_backward(d_llr, batch, cfg, iterations, d_alpha, d_beta, clip, detach, d_ck_lq, d_ck_lr, d_g_final,
                        d_g_iter, d_g_llr, d_g_alpha, d_g_beta, stream, false);
}

int32_t nrldpc_train_forward_f64(const double* d_llr, int32_t batch, const ldpc_in_config_t* cfg,
                                 int32_t iterations, const double* d_alpha, const double* d_beta, double clip,
                                 double* d_final, double* d_iter, double* d_ck_lq, uint32_t* d_ck_lr, void* stream) {
  return train_forward(d_llr, batch, cfg, iterations, d_alpha, d_beta, clip, d_final, d_iter, d_ck_lq, d_ck_lr, stream,
                       true);
}

int32_t nrldpc_train_backward_f64(const double* d_llr, int32_t batch, const ldpc_in_config_t* cfg,
                                  int32_t iterations, const double* d_alpha, const double* d_beta, double clip,
                                  int32_t detach, const double* d_ck_lq, const uint32_t* d_ck_lr,
                                  const double* d_g_final, const double* d_g_iter, double* d_g_llr,
                                  double* d_g_alpha, double* d_g_beta, void* stream) {
  return train_backward(d_llr, batch, cfg, iterations, d_alpha, d_beta, clip, detach, d_ck_lq, d_ck_lr, d_g_final,
                        d_g_iter, d_g_llr, d_g_alpha, d_g_beta, stream, true);
}

int32_t nrldpc_train_checkpoint_words(const ldpc_in_config_t* cfg, int32_t iterations, int32_t batch,
                                      int32_t f64, int64_t* lq_elems, int64_t* msg_words) {
  TrainParams p;
  int block, smem_f, smem_b;
  const int rc = make_train_params(cfg, iterations, batch, 0.0, f64 != 0, &p, &block, &smem_f, &smem_b);
  if (rc != NRLDPC_OK) return rc;
  if (lq_elems) *lq_elems = (int64_t)iterations * batch * p.n;
  if (msg_words) *msg_words = (int64_t)iterations * batch * p.R * p.msg_words;
  return NRLDPC_OK;
}

}  // extern "C"
