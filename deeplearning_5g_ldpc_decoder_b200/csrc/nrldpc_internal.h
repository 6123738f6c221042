// nrldpc_internal.h — definitions shared by the host glue and the CUDA kernels.
#pragma once

#include <stdint.h>

#include <vector>

#include <vector_types.h>

#include "nrldpc_b200.h"

namespace nrldpc {

constexpr int kMaxRows = NRLDPC_BG1_ROWS;   // 46
constexpr int kMaxCols = NRLDPC_BG1_COLS;   // 68
constexpr int kMaxNnz = NRLDPC_BG1_NNZ;     // 316
constexpr int kMaxDegree = NRLDPC_MAX_DEGREE;
constexpr int kMaxZc = NRLDPC_MAX_ZC;
constexpr int kMaxB = 8448;                  // BG1 K at Zc=384
constexpr int kThreadsTarget = 384;          // lifted rows handled by one CTA
constexpr int kMaxGroups = kThreadsTarget / 2;  // Zc=2 packs 192 groups

// One base graph with its CSR view (reference layout, for gen_ldpc_parameters)
// and per-row degrees.
struct BaseGraph {
  int bgn, rows, cols, nnz;
  uint16_t row_off[kMaxRows + 1];
  uint16_t col[kMaxNnz];
  uint16_t vij[8][kMaxNnz];
  uint8_t degree[kMaxRows];
};

const BaseGraph& base_graph(int bgn);

// Everything derived from ldpc_in_config_t that the kernels need.
struct CodeParams {
  int bgn, A, crctype, E, rv, Qm, harq_on;
  int B, Zc, iLS, K, F, N, k0;
  int rows, cols, nnz;
  int lq_len;     // N + 2*Zc = cols*Zc
  int Nv;         // N - F, non-filler positions of the circular buffer
  int c0;         // start position k0 mapped into the compacted buffer
  int symbols;    // E / Qm
  int crc_w;      // 16 or 24
};

// Restatement of gen_ldpc_parameters' validation and derivation
// (c_lib/ldpc_internal.c:66-170).  Returns 0 on success, -1 on a bad config.
int derive_params(const ldpc_in_config_t& in, CodeParams* out, bool verbose);

// Host CRC remainder (c_lib/nr_crc.c:129-179 semantics).
uint32_t crc_remainder(const uint8_t* data, int len, int crctype);

// T[d] = x^(d + W) mod g(x) for d in [0, kMaxB): the CRC remainder of a
// message whose only set bit sits d positions before its end.
void crc_position_table(int crctype, uint32_t* out /* kMaxB */);

// Scratch planes (kThreadsTarget words each) of one lifted check row of degree
// d in the fixed-point kernels: the two minima, the flip bits and the min2
// bits, plus a fifth word for degree-19 rows (layout in nrldpc_fixed_row.cuh).
inline int fixed_row_planes(int d) { return d > 16 ? 5 : 4; }
// Scratch words per CTA of the mixed-size kernel: the larger of the two base
// graphs' layouts (all rows' planes x kThreadsTarget).
uint32_t mixed_scratch_words_per_cta();

// ceil(2^32 / Qm), the constant that turns e / Qm into one high multiply in the
// kernels' scatter-form rate recovery (div_qm); 0 for Qm = 1, whose quotient is
// e itself (its constant, 2^32, does not fit 32 bits).
#ifdef __CUDACC__
__host__ __device__
#endif
inline uint32_t qm_magic(int qm) {
  return qm <= 1 ? 0u : (uint32_t)((0x100000000ull + (uint64_t)qm - 1) / (uint64_t)qm);
}

// Check-node arithmetic of the fixed-point kernels (template parameter kClip):
//  * kClipClamp: clip(rel + msg) is a clamp to [min_llr, max_llr];
//  * kClipDegen: min_llr > max_llr, where the reference's clip is not a clamp
//    (exact int32 arithmetic);
//  * kClipOpenMax: max_llr = 32767 and, in every layer, alpha >= 0 and
//    beta = 0 (algos 1 and 3): the minima need no clip, the offset step is the
//    identity, the scaled minima lie in [0, 32766], and the clamp of the new
//    beliefs is a max with min_llr.  This is the reference's default decoder
//    row.
// `ab` holds each layer's packed alpha | beta << 16 as the kernels read it.
enum { kClipClamp = 0, kClipDegen = 1, kClipOpenMax = 2 };
inline int fixed_clip_mode(const ldpc_decoder_cfg_t& dc, const uint32_t* ab, int rows) {
  if (dc.min_llr > dc.max_llr) return kClipDegen;
  if ((dc.algo != 1 && dc.algo != 3) || dc.max_llr != 32767) return kClipClamp;
  for (int r = 0; r < rows; ++r)
    if ((ab[r] >> 15) != 0u) return kClipClamp;   // alpha < 0 (bit 15) or beta != 0 (bits 16-31)
  return kClipOpenMax;
}

// Alpha/beta per (iteration, row): alpha in the low 16 bits, beta in the high.
inline uint32_t pack_ab(int16_t alpha, int16_t beta) {
  return (uint32_t)(uint16_t)alpha | ((uint32_t)(uint16_t)beta << 16);
}

// Launch parameters of every decode kernel.  Passed by value as a
// __grid_constant__ kernel parameter so that the per-edge tables are read
// through the constant cache with warp-uniform indices.
struct DecodeParams {
  int32_t Zc, R, lq_len, B, K, F, N, Nv, E, Qm, symbols, c0, max_it;
  int32_t G;      // codeword slots per CTA: pairs (fixed point) or codewords (float)
  int32_t nact;   // active threads per CTA = G * Zc
  int32_t num_cw, num_items;
  int32_t harq_on;
  int32_t fill, max_llr, min_llr;
  int32_t weights_T;   // 0: use w_inline[row]; >0: weights[min(it,T-1)*R + row]
  int32_t rr_scatter;  // rate recovery in scatter form (E <= Nv: no LLR repeats)
  int32_t rr_vec;      // LLR rows 16-byte aligned: 8 LLRs per load in the scatter form
  uint32_t qm_magic;   // ceil(2^32 / Qm): e / Qm as __umulhi(e, qm_magic) for e < 2^16
  uint32_t one;        // 1: an add written as a multiply-add by this launch value issues on the FMA pipe
  float f_alpha, f_beta, f_max, f_min;
  const uint32_t* weights;
  const uint32_t* crc_tab;
  const int16_t* llr;
  int64_t llr_stride;
  uint8_t* bits;
  int64_t bits_stride;
  int32_t* status;
  int32_t* iters;
  void* app;
  int64_t app_stride;
  int16_t* harq;
  int64_t harq_stride;
  uint32_t* scratch;
  int64_t scratch_words;   // per CTA
  int32_t* cursor;         // work queue [head, finished CTAs]: zero at launch, rewound by the kernel's
                           // last CTA (null: fixed work items)
  // Per edge: (base column * Zc) in the low 16 bits, (V_ij mod Zc) in the high.
  uint32_t edge[kMaxNnz];
  // The same two fields as byte offsets of 32-bit shared-memory words
  // {base column * Zc * 4, (V_ij mod Zc) * 4}, used by the fixed-point kernel.
  uint2 edge_cs4[kMaxNnz];
  uint32_t lr_off[kMaxRows + 1];   // per-layer word offset inside a CTA's scratch
  uint32_t w_inline[kMaxRows];
  uint16_t row_off[kMaxRows + 1];
};

// Launch parameters of the batched encoder (one CTA per code block).
struct EncodeParams {
  int32_t bgn, Zc, R, cols, A, B, K, F, N, Nv, E, Qm, symbols, c0, Kb;
  int32_t shift0, shift1;   // core-parity circulant shifts (mod Zc): I1/I3 and I2/I4
  int32_t num_cw;
  const uint32_t* crc_tab;  // T[d] of the CRC type
  const uint8_t* info;      // [num_cw][info_stride] payload bytes (A/8 used)
  int64_t info_stride;
  uint8_t* rm;              // [num_cw][rm_stride] rate-matched bytes (ceil(E/8) written)
  int64_t rm_stride;
  uint32_t edge[kMaxNnz];   // base column in the low 16 bits, V_ij mod Zc in the high
  uint16_t row_off[kMaxRows + 1];
};

// ---- mixed-size batches (one persistent kernel, work queue) ----
// Base-graph tables of one (BG, Zc), staged into shared memory per work item.
struct MixedGraph {
  int32_t bgn, Zc, R, lq_len, G, K, N, pad0, pad1;
  uint32_t lr_off[kMaxRows + 1];       // scratch plane offsets, plane stride kThreadsTarget
  uint16_t row_off[kMaxRows + 1];
  uint16_t pad2;
  uint2 edges[kMaxNnz];                // {col*Zc*4, (V mod Zc)*4}
};
// Per code block: its own rate-recovery / CRC parameters and I/O offsets.
struct MixedCw {
  int32_t B, E, Qm, symbols, c0, Nv, F, crctype;
  int64_t llr_off;    // elements into the LLR arena
  int64_t bits_off;   // bytes into the hard-bit arena
  int32_t ncb;        // circular-buffer length (N unless limited-buffer rate matching)
  int32_t harq_mode;  // bit 0: add to the stored soft buffer, bit 1: store the soft buffer
  int64_t harq_off;   // elements into the soft-buffer arena (N + 2Zc of them), when harq_mode != 0
};
// One work item: a CTA's claim on the blocks of one (BG, Zc).  The CTA takes
// up to 2G blocks from that graph's queue and refills each int16 half lane from
// the same queue as soon as its block finishes.
struct MixedItem {
  int32_t graph, pad0, pad1, pad2;
};
struct MixedParams {
  const MixedGraph* graphs;
  const MixedItem* items;
  const int32_t* cb_list;              // blocks grouped by graph: cb_list[key_base[k] .. + key_count[k])
  const int32_t* key_base;             // per graph
  const int32_t* key_count;            // per graph (device-built when num_items_dev is set)
  int32_t* key_cursor;                 // per graph: next unclaimed entry, zeroed before each launch
  const MixedCw* cws;
  int32_t num_items;
  const int32_t* num_items_dev;        // when set, the item count is read from the device (built there)
  int32_t* counter;                    // work-queue head, zeroed before each launch
  const int16_t* llr;
  uint8_t* bits;
  int32_t* status;
  int32_t* iters;
  int16_t* harq;                       // soft-buffer arena of the blocks with harq_mode != 0 (nullable)
  const uint32_t* crc_tab;             // [4][kMaxB]
  uint32_t* scratch;
  int64_t scratch_words;               // per CTA
  int32_t max_it, fill, max_llr, min_llr;
  uint32_t one;                        // 1 (see DecodeParams::one)
  uint32_t w_inline[2][kMaxRows];      // alpha|beta<<16 per row, per base graph (algos 1, 3)
  const uint32_t* weights[2];          // algo 2 tables per base graph
  int32_t weights_T[2];
};

// ---- differentiable unrolled float min-sum (training) ----
struct TrainParams {
  int32_t Zc, R, n, G, nnz, T, batch, detach;
  int32_t alias;              // backward: LQ and dLQ share one shared-memory array per block
  int32_t msg_words;          // 32-bit words of compressed messages per lifted row block (4 Zc f32, 6 Zc f64)
  double clip;                // +inf when LLRs are not clipped
  // Real = float or double, per the entry point.
  const void* llr;            // Real [batch][n] decoder-layout input LLRs
  const void* alpha;          // Real [T][R]
  const void* beta;           // Real [T][R]
  void* final_llr;            // Real [batch][n]
  void* iter_llr;             // Real [T][batch][n] or null
  void* ck_lq;                // Real [T][batch][n] LQ at the start of each iteration
  uint32_t* ck_lr;            // [T][batch][R][msg_words]: Real m1[Zc], m2[Zc]; u32 flips[Zc], first-min index[Zc]
  const void* g_final;        // Real [batch][n] or null
  const void* g_iter;         // Real [T][batch][n] or null
  void* g_llr;                // Real [batch][n]
  void* g_alpha;              // Real [T][R], accumulated
  void* g_beta;               // Real [T][R], accumulated
  void* tape;                 // per CTA: G * nnz * Zc Real
  void* carry;                // per CTA: G * nnz * Zc Real
  int64_t scratch_per_cta;    // elements of tape (and of carry) per CTA
  uint32_t edge[kMaxNnz];     // base column * Zc in the low 16 bits, V mod Zc in the high
  uint16_t row_off[kMaxRows + 1];
};

// Kernel launchers (defined in the .cu files).  Return a cudaError_t value.
int launch_encode(const EncodeParams& p, void* stream);
int launch_train_forward(const TrainParams& p, bool f64, int grid, int block, int smem, void* stream);
int launch_train_backward(const TrainParams& p, bool f64, int grid, int block, int smem, void* stream);
int occupancy_train(bool backward, bool f64, bool bg2, int block, int smem, bool alias = false);
// Mixed-size kernel classes: 0 = 384 threads per CTA (all of them active at
// most), 1 = 256 threads with at most 240 active, three CTAs per SM.  A graph
// of a class holds G = floor(capacity / Zc) lane pairs per CTA.
constexpr int kMixedClasses = 2;
int mixed_class_capacity(int cls);
int launch_mixed(const MixedParams& p, int grid, int clip_mode, void* stream, int cls = 0);
int prepare_mixed(int clip_mode, int cls = 0);
int occupancy_mixed(int clip_mode, int cls = 0);
int launch_channel(const uint8_t* rm, int64_t rm_stride, int32_t num_cw, int32_t E, int32_t Qm, float nv,
                   float sigma, float A, uint64_t seed, int16_t* llr, int64_t llr_stride, float* symbols,
                   void* stream);
int launch_fixed(const DecodeParams& p, int grid, int block, int smem, int clip_mode, void* stream);
int launch_float_minsum(const DecodeParams& p, int grid, int block, int smem, void* stream);
int launch_float_bp(const DecodeParams& p, int grid, int block, int smem, void* stream);

// Occupancy helpers (per kernel variant).
int occupancy_fixed(int block, int smem, int clip_mode, bool refill = false);
int occupancy_float_minsum(int block, int smem);
int occupancy_float_bp(int block, int smem);

void count_launch();

// Current algo-3 degree table entry and algo-2 table (copy); the latter
// returns a generation number that changes whenever the table is replaced.
int16_t current_degree_alpha(int deg);
int device_crc_table(const uint32_t** tab);
int device_trained_table(int bgn, const uint32_t** ptr, int* T);
uint64_t current_trained_table(int bgn, std::vector<uint32_t>* ab, int* T);

}  // namespace nrldpc
