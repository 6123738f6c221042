// nrldpc_noalloc.cu — a decode entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: real-time receive
// pipelines that must not pay cudaMalloc's implicit device synchronisation and
// unbounded latency in the middle of a slot, and host frameworks that own all
// device memory (their own pool or budget) and forbid plug-ins from allocating
// behind their back.  nrldpc_decode_batch_noalloc serves them: it runs the same
// fixed-point decode kernel as nrldpc_decode_batch (algos 1, 2, 3), but its
// message scratch, CRC table and algo-2 table live in file-scope
// `static __device__` arrays that are part of the library image.  The caller
// still provides every input and output buffer.
//
// Costs and rules:
//  * every GPU that loads this library holds the arrays (kNoAllocScratchBytes
//    of scratch plus ~150 KB of tables) until the process exits;
//  * the scratch bounds the number of CTAs in flight, so large batches run as
//    more work items per CTA (slower than nrldpc_decode_batch, same results);
//  * the first call on a device does the set-up for that device (symbol
//    addresses, CRC table upload), so make that first call before any stream
//    capture; likewise the first algo-2 call after nrldpc_set_trained_weights
//    changed a table copies the new table from host memory, so make that call
//    before any capture too;
//  * all calls share the arrays: calls that overlap on the GPU (different
//    streams, or concurrent host threads) race on the scratch and must be
//    serialised by the caller.  Nothing needs clearing between calls: the
//    kernel never reads a message slot before writing it in the same call.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;   // 32 MiB
constexpr int kNoAllocMaxTrainedIters = 64;                   // algo-2 table rows

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchBytes / sizeof(uint32_t)];
static __device__ __align__(256) uint32_t g_noalloc_crc[4 * kMaxB];
static __device__ __align__(256) uint32_t g_noalloc_trained[2][kNoAllocMaxTrainedIters * kMaxRows];

struct NoAllocDevice {
  bool ready = false;
  uint32_t* scratch = nullptr;
  uint32_t* crc = nullptr;
  uint32_t* trained = nullptr;       // [2][kNoAllocMaxTrainedIters * kMaxRows]
  uint64_t trained_gen[2] = {0, 0};
  int num_sms = 0;
};

std::mutex g_na_mu;
std::map<int, NoAllocDevice> g_na_dev;

// Once per device, with that device current: resolve the device addresses of
// the static arrays (host code only sees host-side stand-ins under their names)
// and upload the CRC position table.
int setup_device(NoAllocDevice** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return NRLDPC_ERR_CUDA;
  NoAllocDevice& d = g_na_dev[dev];
  if (!d.ready) {
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&d.scratch), g_noalloc_scratch) != cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&d.crc), g_noalloc_crc) != cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&d.trained), g_noalloc_trained) != cudaSuccess) {
      fprintf(stderr, "nrldpc_decode_batch_noalloc: cudaGetSymbolAddress failed\n");
      return NRLDPC_ERR_CUDA;
    }
    std::vector<uint32_t> tab((size_t)4 * kMaxB);
    for (int t = 0; t < 4; ++t) crc_position_table(t, tab.data() + (size_t)t * kMaxB);
    if (cudaMemcpyToSymbol(g_noalloc_crc, tab.data(), tab.size() * sizeof(uint32_t)) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    if (cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    d.ready = true;
  }
  *out = &d;
  return NRLDPC_OK;
}

}  // namespace
}  // namespace nrldpc

using namespace nrldpc;

extern "C" int32_t nrldpc_decode_batch_noalloc(const int16_t* d_llr, int64_t llr_stride, int32_t num_cw,
                                               const ldpc_in_config_t* inconfig,
                                               const ldpc_decoder_cfg_t* dc, uint8_t* d_bits,
                                               int64_t bits_stride, int32_t* d_status, int32_t* d_iters,
                                               void* d_app, int64_t app_stride, int16_t* d_harq,
                                               int64_t harq_stride, void* stream) {
  if (!inconfig || !dc || num_cw < 0) return NRLDPC_ERR_ARG;
  CodeParams cp;
  if (derive_params(*inconfig, &cp, true) != 0) return NRLDPC_ERR_CONFIG;
  if (dc->algo < 1 || dc->algo > 3) {
    fprintf(stderr, "nrldpc_decode_batch_noalloc: algo %u not supported (fixed-point algos 1-3 only)\n", dc->algo);
    return NRLDPC_ERR_ALGO;
  }
  if (num_cw == 0) return NRLDPC_OK;
  if (!d_llr || llr_stride < cp.E) return NRLDPC_ERR_ARG;
  if (d_bits && bits_stride < (cp.B + 7) / 8) return NRLDPC_ERR_ARG;
  if (d_app && app_stride < cp.lq_len) return NRLDPC_ERR_ARG;
  if (d_harq && harq_stride < cp.lq_len) return NRLDPC_ERR_ARG;

  std::lock_guard<std::mutex> lock(g_na_mu);
  NoAllocDevice* nd = nullptr;
  int rc = setup_device(&nd);
  if (rc != NRLDPC_OK) return rc;

  DecodeParams p;
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
  p.max_it = dc->max_iterations;
  p.rr_scatter = cp.E <= cp.Nv;
  p.qm_magic = qm_magic(cp.Qm);
  p.one = 1u;
  p.harq_on = cp.harq_on;
  p.fill = dc->filling_bit_value;
  p.max_llr = dc->max_llr;
  p.min_llr = dc->min_llr;
  p.crc_tab = nd->crc + (size_t)cp.crctype * kMaxB;
  for (int e = 0; e < g.nnz; ++e) {
    const uint32_t colbase = (uint32_t)g.col[e] * (uint32_t)cp.Zc;
    const uint32_t sh = (uint32_t)(g.vij[cp.iLS][e] % cp.Zc);
    p.edge[e] = colbase | (sh << 16);
    p.edge_cs4[e] = make_uint2(4u * colbase, 4u * sh);
  }
  for (int r = 0; r <= g.rows; ++r) p.row_off[r] = g.row_off[r];
  p.G = std::max(1, kThreadsTarget / cp.Zc);
  p.nact = p.G * cp.Zc;
  p.num_cw = num_cw;
  p.num_items = ((num_cw + 1) / 2 + p.G - 1) / p.G;
  const int16_t alpha = (int16_t)dc->alpha, beta = (int16_t)dc->beta;
  if (dc->algo == 1) {
    for (int r = 0; r < g.rows; ++r) p.w_inline[r] = pack_ab(alpha, beta);
  } else if (dc->algo == 3) {
    for (int r = 0; r < g.rows; ++r) p.w_inline[r] = pack_ab(current_degree_alpha(g.degree[r]), beta);
  } else {
    std::vector<uint32_t> ab;
    int T = 0;
    const uint64_t gen = current_trained_table(cp.bgn, &ab, &T);
    if (T > kNoAllocMaxTrainedIters) {
      fprintf(stderr, "nrldpc_decode_batch_noalloc: algo-2 table has %d iterations, more than the %d this entry "
              "point holds\n", T, kNoAllocMaxTrainedIters);
      return NRLDPC_ERR_ARG;
    }
    const int k = cp.bgn == 1 ? 0 : 1;
    uint32_t* dst = nd->trained + (size_t)k * kNoAllocMaxTrainedIters * kMaxRows;
    if (nd->trained_gen[k] != gen) {
      // Stream-ordered after earlier calls on this stream.  A copy from pageable
      // host memory has read its source by the time it returns, so `ab` may go
      // out of scope without a host synchronisation.
      if (cudaMemcpyAsync(dst, ab.data(), ab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                          reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
        return NRLDPC_ERR_CUDA;
      nd->trained_gen[k] = gen;
    }
    p.weights = dst;
    p.weights_T = T;
  }
  uint32_t off = 0;
  for (int r = 0; r < g.rows; ++r) {
    p.lr_off[r] = off;
    off += (uint32_t)fixed_row_planes(g.degree[r]) * (uint32_t)kThreadsTarget;
  }
  p.lr_off[g.rows] = off;
  p.scratch_words = off;
  const size_t per_cta = (size_t)off * sizeof(uint32_t);
  if (per_cta > kNoAllocScratchBytes) {
    fprintf(stderr, "nrldpc_decode_batch_noalloc: %zu bytes of scratch per CTA exceed the %zu-byte static array\n",
            per_cta, kNoAllocScratchBytes);
    return NRLDPC_ERR_ARG;
  }
  const int clip = fixed_clip_mode(*dc, p.w_inline, g.rows);
  const int block = (p.nact + 31) & ~31;
  const int smem = p.G * cp.lq_len * 4;
  int occ = occupancy_fixed(block, smem, clip);
  if (occ < 1) occ = 1;
  const int fit = (int)(kNoAllocScratchBytes / per_cta);
  const int grid = std::max(1, std::min({p.num_items, occ * nd->num_sms, fit}));
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
  p.scratch = nd->scratch;
  if (launch_fixed(p, grid, block, smem, clip, stream) != 0) return NRLDPC_ERR_CUDA;
  return NRLDPC_OK;
}
