// nrldpc_mixed_api.cu — host side of mixed-size batches: the plan (one block
// queue per (BG, Zc), work items claiming them, device tables), its CUDA
// graph, and a small autotuner over the CTA class of each lifting size
// (code blocks per CTA), the launch shape and the work-item order.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <utility>
#include <vector>

#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

constexpr int kMixedAutotuneCandidates = NRLDPC_MIXED_AUTOTUNE_CANDIDATES;

struct MixedPlanImpl {
  int device = 0;
  int num_cw = 0;
  int num_sms = 0;
  int clip = kClipClamp;   // check-node arithmetic variant (fixed_clip_mode)
  std::vector<MixedGraph> graphs;
  std::vector<std::vector<int>> members;   // block indices per graph, in queue order
  std::vector<MixedCw> cws;
  MixedGraph* d_graphs = nullptr;
  MixedCw* d_cws = nullptr;
  MixedItem* d_items = nullptr;
  int32_t* d_queue = nullptr;     // block queues: cb_list, then key_base, key_count
  int32_t* d_counter = nullptr;   // work-item head, then one cursor per graph
  uint32_t* d_scratch = nullptr;
  uint32_t* d_scratch1 = nullptr;   // class-1 scratch (the classes may run at the same time)
  int scratch1_ctas = 0;
  cudaStream_t side = nullptr;      // class-1 launches, forked from and joined to the caller's stream
  cudaEvent_t fork = nullptr, join = nullptr;
  size_t items_cap = 0;
  int scratch_ctas = 0;
  MixedParams params = {};   // class-0 launch; the class-1 launch differs in items and head counter
  int order = 0;          // 0: largest work first, 1: graphs interleaved
  int cls_mode = 0;       // 0: every graph in class 0; 1: each graph in the class that keeps more rows active
  int ctas_per_sm = 2;    // class 0 (class 1 runs at its occupancy, 3 per SM)
  std::vector<int> cls;   // per graph
  int num_items_c[kMixedClasses] = {0, 0};
  int grid_c[kMixedClasses] = {0, 0};
  int grid = 1;
  // captured graph
  cudaGraphExec_t exec = nullptr;
  const void* cap_ptrs[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaStream_t cap_stream = nullptr;
  int cap_order = -1, cap_ctas = -1, cap_mode = -1;
};


void free_plan(MixedPlanImpl* pl) {
  if (pl->exec) cudaGraphExecDestroy(pl->exec);
  cudaFree(pl->d_graphs);
  cudaFree(pl->d_cws);
  cudaFree(pl->d_items);
  cudaFree(pl->d_queue);
  cudaFree(pl->d_counter);
  cudaFree(pl->d_scratch);
  cudaFree(pl->d_scratch1);
  if (pl->fork) cudaEventDestroy(pl->fork);
  if (pl->join) cudaEventDestroy(pl->join);
  if (pl->side) cudaStreamDestroy(pl->side);
  delete pl;
}

}  // namespace

uint32_t mixed_scratch_words_per_cta() {
  uint32_t best = 0;
  for (int bgn = 1; bgn <= 2; ++bgn) {
    const BaseGraph& g = base_graph(bgn);
    uint32_t planes = 0;
    for (int r = 0; r < g.rows; ++r) planes += (uint32_t)fixed_row_planes(g.degree[r]);
    best = std::max(best, planes * (uint32_t)kThreadsTarget);
  }
  return best;
}

namespace {

MixedGraph make_graph(int bgn, int Zc, int iLS, int cap) {
  MixedGraph m;
  memset(&m, 0, sizeof(m));
  const BaseGraph& g = base_graph(bgn);
  m.bgn = bgn;
  m.Zc = Zc;
  m.R = g.rows;
  m.lq_len = g.cols * Zc;
  m.G = std::max(1, cap / Zc);
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

// Work items for the current order: per graph, one claim per G lane pairs of
// its blocks (a CTA refills its lanes from the graph's queue, so a claim may
// end up with more blocks than 2G or, when other CTAs drained the queue, none).
// The items of class-0 graphs come first, then those of class-1 graphs.
int build_items(MixedPlanImpl* pl) {
  struct It {
    MixedItem m;
    double cost;
    int graph_rank;
  };
  std::vector<It> all;
  for (int c = 0; c < kMixedClasses; ++c) {
  std::vector<It> items;
  for (size_t gi = 0; gi < pl->graphs.size(); ++gi) {
    if (pl->cls[gi] != c) continue;
    const MixedGraph& g = pl->graphs[gi];
    const BaseGraph& bg = base_graph(g.bgn);
    const int npairs_total = ((int)pl->members[gi].size() + 1) / 2;
    int rank = 0;
    for (int p0 = 0; p0 < npairs_total; p0 += g.G, ++rank) {
      It it;
      memset(&it.m, 0, sizeof(it.m));
      it.m.graph = (int32_t)gi;
      it.cost = (double)bg.nnz * g.Zc * std::min(g.G, npairs_total - p0);
      it.graph_rank = rank;
      items.push_back(it);
    }
  }
  if (pl->order == 0) {
    std::stable_sort(items.begin(), items.end(), [](const It& a, const It& b) { return a.cost > b.cost; });
  } else {
    std::stable_sort(items.begin(), items.end(), [](const It& a, const It& b) { return a.graph_rank < b.graph_rank; });
  }
  pl->num_items_c[c] = (int)items.size();
  all.insert(all.end(), items.begin(), items.end());
  }
  std::vector<MixedItem> host(all.size());
  for (size_t i = 0; i < all.size(); ++i) host[i] = all[i].m;
  if (host.size() > pl->items_cap) {
    cudaFree(pl->d_items);
    if (cudaMalloc(&pl->d_items, host.size() * sizeof(MixedItem)) != cudaSuccess) return NRLDPC_ERR_CUDA;
    pl->items_cap = host.size();
  }
  if (cudaMemcpy(pl->d_items, host.data(), host.size() * sizeof(MixedItem), cudaMemcpyHostToDevice) != cudaSuccess)
    return NRLDPC_ERR_CUDA;
  pl->params.items = pl->d_items;
  pl->params.num_items = (int32_t)pl->num_items_c[0];
  return NRLDPC_OK;
}

// Class of graph (BG, Zc) in cls_mode 1: the one that keeps more lifted rows
// active per SM (class 0: 2 CTAs of floor(384/Zc) x Zc rows; class 1: 3 CTAs of
// floor(240/Zc) x Zc rows).
int natural_class(int Zc) {
  const int cap1 = mixed_class_capacity(1), cap0 = mixed_class_capacity(0);
  if (Zc > cap1) return 0;
  return 3 * (cap1 / Zc) * Zc > 2 * (cap0 / Zc) * Zc ? 1 : 0;
}

int configure(MixedPlanImpl* pl, int ctas_per_sm, int order, int cls_mode) {
  const bool regraph = cls_mode != pl->cls_mode || pl->cls.empty();
  if (regraph) {
    pl->cls_mode = cls_mode;
    pl->cls.assign(pl->graphs.size(), 0);
    for (size_t gi = 0; gi < pl->graphs.size(); ++gi) {
      const int c = cls_mode == 1 ? natural_class(pl->graphs[gi].Zc) : 0;
      pl->cls[gi] = c;
      pl->graphs[gi].G = std::max(1, mixed_class_capacity(c) / pl->graphs[gi].Zc);
    }
    if (cudaMemcpy(pl->d_graphs, pl->graphs.data(), pl->graphs.size() * sizeof(MixedGraph),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
  }
  if (regraph || order != pl->order || !pl->params.items) {
    pl->order = order;
    const int rc = build_items(pl);
    if (rc != NRLDPC_OK) return rc;
  }
  int occ = occupancy_mixed(pl->clip, 0);
  if (occ < 1) occ = 1;
  int occ1 = occupancy_mixed(pl->clip, 1);
  if (occ1 < 1) occ1 = 1;
  pl->ctas_per_sm = std::max(1, std::min(ctas_per_sm, occ));
  pl->grid_c[0] = std::max(0, std::min(pl->num_items_c[0], pl->ctas_per_sm * pl->num_sms));
  pl->grid_c[1] = std::max(0, std::min(pl->num_items_c[1], occ1 * pl->num_sms));
  pl->grid = std::max(1, pl->grid_c[0]);
  if (pl->grid_c[1] > pl->scratch1_ctas) {
    cudaFree(pl->d_scratch1);
    pl->d_scratch1 = nullptr;
    if (cudaMalloc(&pl->d_scratch1, (size_t)pl->grid_c[1] * mixed_scratch_words_per_cta() * sizeof(uint32_t)) !=
        cudaSuccess)
      return NRLDPC_ERR_CUDA;
    pl->scratch1_ctas = pl->grid_c[1];
  }
  if (pl->grid > pl->scratch_ctas) {
    cudaFree(pl->d_scratch);
    pl->d_scratch = nullptr;
    if (cudaMalloc(&pl->d_scratch, (size_t)pl->grid * mixed_scratch_words_per_cta() * sizeof(uint32_t)) != cudaSuccess)
      return NRLDPC_ERR_CUDA;
    pl->scratch_ctas = pl->grid;
  }
  pl->params.scratch = pl->d_scratch;
  return NRLDPC_OK;
}

int enqueue(MixedPlanImpl* pl, cudaStream_t s) {
  // both classes' work-item heads and every graph's queue cursor start at zero
  if (cudaMemsetAsync(pl->params.counter, 0, sizeof(int32_t) * (kMixedClasses + pl->graphs.size()), s) !=
      cudaSuccess)
    return NRLDPC_ERR_CUDA;
  // The class-1 launch runs beside the class-0 one on a side stream (fork and
  // join through events, which a CUDA graph capture records as a fork/join):
  // its CTAs take the SMs that class-0 CTAs leave as their queue drains, so the
  // two classes do not each pay a tail.  The graphs of the two classes are
  // disjoint; each class has its own items, head counter and scratch.
  const bool both = pl->grid_c[0] > 0 && pl->grid_c[1] > 0;
  if (both && (cudaEventRecord(pl->fork, s) != cudaSuccess || cudaStreamWaitEvent(pl->side, pl->fork, 0) != cudaSuccess))
    return NRLDPC_ERR_CUDA;
  if (pl->grid_c[0] > 0 && launch_mixed(pl->params, pl->grid_c[0], pl->clip, s, 0) != 0) return NRLDPC_ERR_CUDA;
  if (pl->grid_c[1] > 0) {
    MixedParams p1 = pl->params;
    p1.items = pl->d_items + pl->num_items_c[0];
    p1.num_items = pl->num_items_c[1];
    p1.counter = pl->params.counter + 1;
    p1.scratch = pl->d_scratch1;
    if (launch_mixed(p1, pl->grid_c[1], pl->clip, both ? pl->side : s, 1) != 0) return NRLDPC_ERR_CUDA;
  }
  if (both && (cudaEventRecord(pl->join, pl->side) != cudaSuccess || cudaStreamWaitEvent(s, pl->join, 0) != cudaSuccess))
    return NRLDPC_ERR_CUDA;
  return NRLDPC_OK;
}

int execute(MixedPlanImpl* pl, const int16_t* llr, uint8_t* bits, int32_t* status, int32_t* iters, bool use_graph,
            cudaStream_t s) {
  pl->params.llr = llr;
  pl->params.bits = bits;
  pl->params.status = status;
  pl->params.iters = iters;
  if (!use_graph || s == nullptr) return enqueue(pl, s);
  const void* ptrs[4] = {llr, bits, status, iters};
  const bool same = pl->exec && s == pl->cap_stream && pl->cap_order == pl->order &&
                    pl->cap_ctas == pl->ctas_per_sm && pl->cap_mode == pl->cls_mode &&
                    memcmp(ptrs, pl->cap_ptrs, sizeof(ptrs)) == 0;
  if (!same) {
    if (pl->exec) cudaGraphExecDestroy(pl->exec);
    pl->exec = nullptr;
    if (prepare_mixed(pl->clip, 0) != 0 || prepare_mixed(pl->clip, 1) != 0) return NRLDPC_ERR_CUDA;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return NRLDPC_ERR_CUDA;
    const int rc = enqueue(pl, s);
    if (cudaStreamEndCapture(s, &graph) != cudaSuccess || rc != NRLDPC_OK) {
      if (graph) cudaGraphDestroy(graph);
      return NRLDPC_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&pl->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return NRLDPC_ERR_CUDA;
    memcpy(pl->cap_ptrs, ptrs, sizeof(ptrs));
    pl->cap_stream = s;
    pl->cap_order = pl->order;
    pl->cap_ctas = pl->ctas_per_sm;
    pl->cap_mode = pl->cls_mode;
  }
  if (cudaGraphLaunch(pl->exec, s) != cudaSuccess) return NRLDPC_ERR_CUDA;
  if (pl->grid_c[0] > 0) count_launch();   // the kernel nodes of the replayed graph
  if (pl->grid_c[1] > 0) count_launch();
  return NRLDPC_OK;
}

}  // namespace
}  // namespace nrldpc

using namespace nrldpc;

extern "C" {

int32_t nrldpc_mixed_plan_create(const nrldpc_block_t* blocks, int32_t num_blocks, const ldpc_decoder_cfg_t* dc,
                                 void** plan_out) {
  if (!plan_out || !dc || num_blocks <= 0 || !blocks) return NRLDPC_ERR_ARG;
  *plan_out = nullptr;
  if (dc->algo < 1 || dc->algo > 3) {
    fprintf(stderr, "nrldpc_mixed_plan_create: fixed-point algos 1-3 only (got %u)\n", dc->algo);
    return NRLDPC_ERR_ALGO;
  }
  MixedPlanImpl* pl = new MixedPlanImpl();
  cudaGetDevice(&pl->device);
  if (cudaStreamCreateWithFlags(&pl->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&pl->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&pl->join, cudaEventDisableTiming) != cudaSuccess) {
    free_plan(pl);
    return NRLDPC_ERR_CUDA;
  }
  if (cudaDeviceGetAttribute(&pl->num_sms, cudaDevAttrMultiProcessorCount, pl->device) != cudaSuccess) {
    free_plan(pl);
    return NRLDPC_ERR_CUDA;
  }
  pl->num_cw = num_blocks;
  std::map<std::pair<int, int>, int> gidx;
  pl->cws.resize(num_blocks);
  for (int i = 0; i < num_blocks; ++i) {
    CodeParams cp;
    if (derive_params(blocks[i].cfg, &cp, true) != 0) {
      free_plan(pl);
      return NRLDPC_ERR_CONFIG;
    }
    if (cp.harq_on || blocks[i].llr_offset < 0 || blocks[i].bits_offset < 0) {
      free_plan(pl);
      return NRLDPC_ERR_ARG;
    }
    const auto key = std::make_pair(cp.bgn, cp.Zc);
    auto itg = gidx.find(key);
    if (itg == gidx.end()) {
      itg = gidx.emplace(key, (int)pl->graphs.size()).first;
      pl->graphs.push_back(make_graph(cp.bgn, cp.Zc, cp.iLS, mixed_class_capacity(0)));
      pl->members.emplace_back();
    }
    pl->members[itg->second].push_back(i);
    MixedCw& c = pl->cws[i];
    c.B = cp.B;
    c.E = cp.E;
    c.Qm = cp.Qm;
    c.symbols = cp.symbols;
    c.c0 = cp.c0;
    c.Nv = cp.Nv;
    c.F = cp.F;
    c.crctype = cp.crctype;
    c.llr_off = blocks[i].llr_offset;
    c.bits_off = blocks[i].bits_offset;
    c.ncb = cp.N;
    c.harq_mode = 0;
    c.harq_off = 0;
  }
  MixedParams& p = pl->params;
  p.max_it = dc->max_iterations;
  p.fill = dc->filling_bit_value;
  p.max_llr = dc->max_llr;
  p.one = 1u;
  p.min_llr = dc->min_llr;
  p.scratch_words = mixed_scratch_words_per_cta();
  for (int b = 0; b < 2; ++b) {
    const BaseGraph& g = base_graph(b + 1);
    for (int r = 0; r < g.rows; ++r) {
      const int16_t alpha = dc->algo == 3 ? current_degree_alpha(g.degree[r]) : (int16_t)dc->alpha;
      p.w_inline[b][r] = pack_ab(alpha, (int16_t)dc->beta);
    }
    p.weights_T[b] = 0;
    if (dc->algo == 2 && device_trained_table(b + 1, &p.weights[b], &p.weights_T[b]) != NRLDPC_OK) {
      free_plan(pl);
      return NRLDPC_ERR_CUDA;
    }
  }
  // open-max arithmetic only when both base graphs' layers qualify
  pl->clip = fixed_clip_mode(*dc, p.w_inline[0], base_graph(1).rows);
  if (pl->clip == kClipOpenMax) pl->clip = fixed_clip_mode(*dc, p.w_inline[1], base_graph(2).rows);
  // per-graph block queues: members of each graph in pairing order
  std::vector<int32_t> queue;
  std::vector<int32_t> base(pl->graphs.size()), count(pl->graphs.size());
  for (size_t gi = 0; gi < pl->graphs.size(); ++gi) {
    base[gi] = (int32_t)queue.size();
    count[gi] = (int32_t)pl->members[gi].size();
    queue.insert(queue.end(), pl->members[gi].begin(), pl->members[gi].end());
  }
  const size_t ng = pl->graphs.size();
  queue.insert(queue.end(), base.begin(), base.end());
  queue.insert(queue.end(), count.begin(), count.end());
  if (device_crc_table(&p.crc_tab) != NRLDPC_OK ||
      cudaMalloc(&pl->d_graphs, pl->graphs.size() * sizeof(MixedGraph)) != cudaSuccess ||
      cudaMalloc(&pl->d_cws, pl->cws.size() * sizeof(MixedCw)) != cudaSuccess ||
      cudaMalloc(&pl->d_counter, sizeof(int32_t) * (kMixedClasses + ng)) != cudaSuccess ||
      cudaMalloc(&pl->d_queue, sizeof(int32_t) * queue.size()) != cudaSuccess ||
      cudaMemcpy(pl->d_graphs, pl->graphs.data(), pl->graphs.size() * sizeof(MixedGraph), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(pl->d_cws, pl->cws.data(), pl->cws.size() * sizeof(MixedCw), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(pl->d_queue, queue.data(), sizeof(int32_t) * queue.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    free_plan(pl);
    return NRLDPC_ERR_CUDA;
  }
  p.cb_list = pl->d_queue;
  p.key_base = pl->d_queue + (queue.size() - 2 * ng);
  p.key_count = pl->d_queue + (queue.size() - ng);
  p.key_cursor = pl->d_counter + kMixedClasses;
  p.graphs = pl->d_graphs;
  p.cws = pl->d_cws;
  p.counter = pl->d_counter;
  pl->cls_mode = -1;   // configure() assigns the classes and uploads the graph tables
  const int rc = configure(pl, 2, 0, 1);
  if (rc != NRLDPC_OK) {
    free_plan(pl);
    return rc;
  }
  *plan_out = pl;
  return NRLDPC_OK;
}

int32_t nrldpc_mixed_plan_execute(void* plan, const int16_t* d_llr, uint8_t* d_bits, int32_t* d_status,
                                  int32_t* d_iterations, int32_t use_graph, void* stream) {
  if (!plan || !d_llr) return NRLDPC_ERR_ARG;
  return execute(static_cast<MixedPlanImpl*>(plan), d_llr, d_bits, d_status, d_iterations, use_graph != 0,
                 reinterpret_cast<cudaStream_t>(stream));
}

// Autotuner candidates: (class mode, class-0 CTAs per SM, work order).
constexpr int kCand[kMixedAutotuneCandidates][3] = {{1, 2, 0}, {1, 1, 0}, {1, 2, 1}, {1, 1, 1},
                                                    {0, 2, 0}, {0, 1, 0}, {0, 2, 1}, {0, 1, 1}};

int32_t nrldpc_mixed_plan_select(void* plan, int32_t candidate) {
  if (!plan || candidate < 0 || candidate >= kMixedAutotuneCandidates) return NRLDPC_ERR_ARG;
  const int* c = kCand[candidate];
  return configure(static_cast<MixedPlanImpl*>(plan), c[1], c[2], c[0]);
}

int32_t nrldpc_mixed_plan_autotune(void* plan, const int16_t* d_llr, uint8_t* d_bits, int32_t* d_status,
                                   int32_t* d_iterations, float* ms_out, void* stream) {
  if (!plan || !d_llr) return NRLDPC_ERR_ARG;
  MixedPlanImpl* pl = static_cast<MixedPlanImpl*>(plan);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const auto& cand = kCand;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return NRLDPC_ERR_CUDA;
  int best = 0;
  float best_ms = 1e30f;
  for (int c = 0; c < kMixedAutotuneCandidates; ++c) {
    if (configure(pl, cand[c][1], cand[c][2], cand[c][0]) != NRLDPC_OK) return NRLDPC_ERR_CUDA;
    if (execute(pl, d_llr, d_bits, d_status, d_iterations, false, s) != NRLDPC_OK) return NRLDPC_ERR_CUDA;
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; ++r)
      if (execute(pl, d_llr, d_bits, d_status, d_iterations, false, s) != NRLDPC_OK) return NRLDPC_ERR_CUDA;
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) return NRLDPC_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= 3.f;
    if (ms_out) ms_out[c] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (configure(pl, cand[best][1], cand[best][2], cand[best][0]) != NRLDPC_OK) return NRLDPC_ERR_CUDA;
  return best;
}

int32_t nrldpc_mixed_plan_destroy(void* plan) {
  if (plan) free_plan(static_cast<MixedPlanImpl*>(plan));
  return NRLDPC_OK;
}

}  // extern "C"
