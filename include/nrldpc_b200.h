/*
 * nrldpc_b200.h — C ABI of the B200 5G NR LDPC receive path.
 *
 * One shared library (deeplearning_5g_ldpc_decoder_b200/libnrldpc_b200.so)
 * exports two groups of entry points:
 *
 *  1. Drop-in replacements for the reference library's C ABI.  Their
 *     signatures, record layouts, argument meaning and return codes are those
 *     of the reference's c_lib/nr_ldpc.h, so the reference's ctypes harness
 *     (scripts/ldpc_c_sim_common.py:60-109) and table loader
 *     (deep_learning/ldpc_table_config.py:93-154) bind them unchanged.
 *
 *  2. Batched, stream-ordered device entry points (nrldpc_*), which take
 *     device pointers and a cudaStream_t and decode many codewords per call.
 *
 * Every decoder entry point runs on the GPU.  There is no CPU fallback: if no
 * CUDA device is usable the calls return NRLDPC_ERR_CUDA (-1).
 *
 * Return codes (mirroring c_lib/c_ldpc_5g_decoder.c:16-32):
 *    0  CRC passed within max_iterations
 *    1  not converged (CRC still failing after max_iterations)
 *   -1  CUDA / runtime error
 *   -2  invalid LDPC configuration
 *   -3  invalid decoder algorithm
 *   -4  invalid argument to a batched entry point (bad pointer / size)
 */
#ifndef NRLDPC_B200_H
#define NRLDPC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NRLDPC_OK 0
#define NRLDPC_NOT_CONVERGED 1
#define NRLDPC_ERR_CUDA (-1)
#define NRLDPC_ERR_CONFIG (-2)
#define NRLDPC_ERR_ALGO (-3)
#define NRLDPC_ERR_ARG (-4)

#define NRLDPC_BG1_ROWS 46
#define NRLDPC_BG1_COLS 68
#define NRLDPC_BG1_NNZ 316
#define NRLDPC_BG2_ROWS 42
#define NRLDPC_BG2_COLS 52
#define NRLDPC_BG2_NNZ 197
#define NRLDPC_MAX_DEGREE 19
#define NRLDPC_MAX_ZC 384

/* Caller-supplied code-block configuration.  Same layout as the reference's
 * ldpc_in_config_t (c_lib/nr_ldpc.h:42-50): seven uint16_t, 14 bytes. */
typedef struct {
    uint16_t bgn;     /* base graph: 1 or 2 */
    uint16_t A;       /* payload bits before CRC (multiple of 8) */
    uint16_t crctype; /* 0 CRC16, 1 CRC24A, 2 CRC24B, 3 CRC24C */
    uint16_t E;       /* rate-matched bits (multiple of Qm) */
    uint16_t rv;      /* redundancy version 0..3 */
    uint16_t Qm;      /* modulation order 1, 2, 4, 6 or 8 */
    uint16_t HARQ_on; /* 1: add to the soft buffer, 0: start a fresh buffer */
} ldpc_in_config_t;

/* Derived parameters.  Same layout as the reference's ldpc_config_t
 * (c_lib/nr_ldpc.h:54-79); the three table pointers point at this library's
 * own copies of the base graph in the reference's CSR form (row offsets,
 * column ids, raw shifts of the selected lifting set). */
typedef struct {
    uint16_t bgn, A, crctype, E, rv, Qm, HARQ_on;
    uint16_t B, Zc, iLS, K, F, N, k0;
    uint16_t *Vij_array;
    uint16_t *HBG_array;
    uint16_t *HBG_offset_array;
} ldpc_config_t;

/* Decoder settings, the row [algo, max_iterations, alpha, beta,
 * filling_bit_value, max_llr, min_llr].  Same layout as the reference's
 * ldpc_decoder_cfg_t (c_lib/nr_ldpc.h:82-90).  alpha and beta are unsigned at
 * the ABI and reinterpreted as int16_t by the fixed-point decoders, exactly
 * as the reference does (c_lib/fixedpoint_ldpc_decoder.c:207-209). */
typedef struct {
    uint16_t algo;           /* 0 BP, 1 min-sum, 2 trained min-sum, 3 degree min-sum, 4 float min-sum */
    uint16_t max_iterations;
    uint16_t alpha;          /* Q15 normalisation */
    uint16_t beta;           /* offset, LLR units (x128 scale) */
    int16_t filling_bit_value;
    int16_t max_llr;
    int16_t min_llr;
} ldpc_decoder_cfg_t;

/* ------------------------------------------------------------------------ */
/* 1. Reference ABI                                                          */
/* ------------------------------------------------------------------------ */

/* Validate a configuration and derive B, Zc, iLS, K, F, N, k0 and the table
 * pointers.  Returns 0 or -1.  Replaces gen_ldpc_parameters
 * (c_lib/nr_ldpc.h:108, c_lib/ldpc_internal.c:66-170). */
int gen_ldpc_parameters(ldpc_config_t *params, ldpc_in_config_t *inconfig);

/* Decode one code block from host memory: rate recovery (with HARQ combining
 * into this library's process-wide soft buffer when HARQ_on=1), layered
 * decoding with the selected algorithm, CRC early termination.  Writes
 * ceil(B/8) bytes of hard decisions, MSB first.  Supports algo 0..4.
 * Replaces cuda_ldpc_5g_decode (CUDA/cuda_ldpc_5g_decoder.cu:31-58), which
 * supports only algo 1 and 4. */
int32_t cuda_ldpc_5g_decode(int16_t *LLr, uint8_t *hardbits,
                            ldpc_in_config_t *inconfig,
                            ldpc_decoder_cfg_t *decoder_config);

/* Same call under the C library's symbol name (c_lib/nr_ldpc.h:127,
 * c_lib/c_ldpc_5g_decoder.c:34-79); it runs on the GPU as well. */
int32_t c_ldpc_5g_decode(int16_t *LLr, uint8_t *hardbits,
                         ldpc_in_config_t *inconfig,
                         ldpc_decoder_cfg_t *decoder_config);

/* Encode one code block from host memory: CRC attach, QC-LDPC encoding, rate
 * matching to E bits with the Qm interleave, packed MSB first into
 * ceil(E/8) bytes of rm_bytes.  Runs on the GPU.  Returns 0, -2 (invalid
 * configuration) or -1 (CUDA error).  Replaces cuda_ldpc_5g_encode
 * (CUDA/cuda_ldpc_5g_encoder.cu:47-84), the symbol the reference's BLER
 * harness binds next to the decoder (scripts/ldpc_c_sim_common.py:76-83). */
int32_t cuda_ldpc_5g_encode(uint8_t *infobytes, uint8_t *rm_bytes,
                            ldpc_in_config_t *inconfig);

/* Same call under the C library's symbol name (c_lib/nr_ldpc.h:129,
 * c_lib/c_ldpc_5g_encoder.c:66-88); it runs on the GPU as well. */
int32_t c_ldpc_5g_encode(uint8_t *infobytes, uint8_t *rm_bytes,
                         ldpc_in_config_t *inconfig);

/* Test channel: unpack num_bits MSB-first bits, NR QAM-map them (Qm 1..8),
 * add complex AWGN of power 10^(noise_power_db/10), max-log demap and
 * quantise round(128*LLR) to +-10000.  Runs on the GPU from host buffers.
 * Same signature, arguments and return codes (0 / -1) as the reference's
 * tx_rx_process (c_lib/nr_ldpc.h:123, c_lib/tx_rx_process.c:286-324); the
 * noise comes from this library's own generator, seeded by
 * nrldpc_channel_seed() instead of srand(). */
int tx_rx_process(const uint8_t *inbytes, size_t num_bits, uint16_t Qm,
                  float noise_power_db, int16_t *llr_out);

/* Table-driven NR CRC remainder over len bytes, MSB first; 0 for an
 * unknown crctype.  Host function.  Replaces calculate_crc
 * (c_lib/nr_ldpc.h:102, c_lib/nr_crc.c:170-179). */
uint32_t calculate_crc(const uint8_t *data, int len, int crctype);

/* ------------------------------------------------------------------------ */
/* 2. Batched device API (no counterpart in the reference, which decodes one */
/*    code block per call)                                                   */
/* ------------------------------------------------------------------------ */

/* Decode num_cw code blocks that share one configuration.
 *
 *   d_llr        device int16 [num_cw][llr_stride], rate-matched order, E used
 *   d_hardbits   device uint8 [num_cw][bits_stride], ceil(B/8) bytes written
 *                (left untouched when max_iterations == 0, as the reference)
 *   d_status     device int32 [num_cw]: 0 CRC pass, 1 not converged (nullable)
 *   d_iterations device int32 [num_cw]: iterations executed (nullable)
 *   d_app        device [num_cw][app_stride] final beliefs LQ, N+2*Zc values:
 *                int16 for algos 1-3, float32 for algos 0 and 4 (nullable)
 *   d_harq       device int16 [num_cw][harq_stride] per-codeword soft buffers
 *                of N+2*Zc values (nullable).  When given, rate recovery starts
 *                from it if inconfig->HARQ_on == 1, and the recovered buffer
 *                is written back to it.
 *   stream       cudaStream_t (NULL = legacy default stream)
 *
 * Stream-ordered: returns after enqueueing.  Scratch memory is owned by the
 * library, one buffer per (device, stream).  Returns 0, -1, -2, -3 or -4. */
int32_t nrldpc_decode_batch(const int16_t *d_llr, int64_t llr_stride,
                            int32_t num_cw,
                            const ldpc_in_config_t *inconfig,
                            const ldpc_decoder_cfg_t *decoder_cfg,
                            uint8_t *d_hardbits, int64_t bits_stride,
                            int32_t *d_status, int32_t *d_iterations,
                            void *d_app, int64_t app_stride,
                            int16_t *d_harq, int64_t harq_stride,
                            void *stream);

/* Same as nrldpc_decode_batch, from and to HOST memory: copies the LLRs in,
 * decodes, copies hard bits / status / iterations back, and returns once they
 * are in host memory (the work starts after what is already queued on
 * `stream`; copies and decodes overlap in chunks on internal streams).
 * Pinned host buffers give full copy bandwidth.  h_status and h_iterations
 * are nullable. */
int32_t nrldpc_decode_batch_host(const int16_t *h_llr, int64_t llr_stride,
                                 int32_t num_cw,
                                 const ldpc_in_config_t *inconfig,
                                 const ldpc_decoder_cfg_t *decoder_cfg,
                                 uint8_t *h_hardbits, int64_t bits_stride,
                                 int32_t *h_status, int32_t *h_iterations,
                                 void *stream);

/* No counterpart in the reference.  The fixed-point decode (algos 1-3) of
 * nrldpc_decode_batch, same arguments and results, for callers that may not
 * allocate device memory: real-time receive pipelines that cannot afford
 * cudaMalloc's device synchronisation and latency mid-slot, and host
 * frameworks that own every device allocation.  It calls no cudaMalloc /
 * cudaFree: its message scratch (32 MiB, bounding the CTAs in flight) and
 * tables are static device arrays of the library, held by every GPU that uses
 * this entry point until the process exits.  The first call on a device
 * resolves those arrays and uploads the CRC table, so make it before any
 * stream capture; the first algo-2 call after nrldpc_set_trained_weights
 * changed a table uploads that table, so make it before any capture too.
 * All calls share the arrays: calls that overlap on the GPU
 * race and must be serialised by the caller.  Returns -3 for algos 0 and 4,
 * -4 if an algo-2 table has more than 64 iterations or a configuration needs
 * more scratch per CTA than the array holds. */
int32_t nrldpc_decode_batch_noalloc(const int16_t *d_llr, int64_t llr_stride,
                                    int32_t num_cw,
                                    const ldpc_in_config_t *inconfig,
                                    const ldpc_decoder_cfg_t *decoder_cfg,
                                    uint8_t *d_hardbits, int64_t bits_stride,
                                    int32_t *d_status, int32_t *d_iterations,
                                    void *d_app, int64_t app_stride,
                                    int16_t *d_harq, int64_t harq_stride,
                                    void *stream);

/* Encode num_cw code blocks of one configuration on the device:
 *   d_info  uint8 [num_cw][info_stride], A/8 payload bytes used
 *   d_rm    uint8 [num_cw][rm_stride], ceil(E/8) rate-matched bytes written
 * Stream-ordered.  No counterpart in the reference (one block per call there).
 * Returns 0, -1, -2 or -4. */
int32_t nrldpc_encode_batch(const uint8_t *d_info, int64_t info_stride,
                            int32_t num_cw, const ldpc_in_config_t *inconfig,
                            uint8_t *d_rm, int64_t rm_stride, void *stream);

/* Same with limited-buffer rate matching (TS 38.212 5.4.2.1): bit selection
 * over a circular buffer of ncb bits (K - 2Zc <= ncb < N; 0 or >= N: N) with
 * k0 computed for it.  Returns 0, -1, -2 or -4. */
int32_t nrldpc_encode_batch_ncb(const uint8_t *d_info, int64_t info_stride,
                                int32_t num_cw, const ldpc_in_config_t *inconfig, int32_t ncb,
                                uint8_t *d_rm, int64_t rm_stride, void *stream);

/* Device LLR front-end for num_cw blocks: d_rm uint8 [num_cw][rm_stride]
 * (ceil(E/8) packed bits used) -> d_llr int16 [num_cw][llr_stride] (E
 * values), through the same mapping / AWGN / demapping / quantisation as
 * tx_rx_process.  The noise of (block, symbol) is a fixed function of seed.
 * d_symbols (nullable) receives the noisy symbols, float [num_cw][E/Qm][2].
 * Stream-ordered.  No counterpart in the reference.  Returns 0, -1 or -4. */
int32_t nrldpc_channel_batch(const uint8_t *d_rm, int64_t rm_stride,
                             int32_t num_cw, int32_t E, int32_t Qm,
                             float noise_power_db, uint64_t seed,
                             int16_t *d_llr, int64_t llr_stride,
                             float *d_symbols, void *stream);

/* Seed of tx_rx_process's noise generator (the reference uses srand()). */
void nrldpc_channel_seed(uint64_t seed);

/* ---- mixed-size batches (no counterpart in the reference) ---- */

/* One code block of a mixed batch: its configuration (HARQ_on must be 0) and
 * where its E LLRs (elements) and ceil(B/8) hard bits (bytes) live in the
 * caller's LLR and output arenas. */
typedef struct {
    ldpc_in_config_t cfg;
    int64_t llr_offset;
    int64_t bits_offset;
} nrldpc_block_t;

/* Plan the decode of num_blocks blocks that may mix base graphs, lifting
 * sizes, E, Qm, rv and CRC types, with one fixed-point decoder setting
 * (algos 1-3).  Blocks of the same (BG, Zc) are paired into int16x2 lanes and
 * grouped into work items that one persistent kernel pulls from a device work
 * queue.  The plan owns its device tables and scratch.  Returns 0, -1, -2,
 * -3 or -4. */
int32_t nrldpc_mixed_plan_create(const nrldpc_block_t *blocks, int32_t num_blocks,
                                 const ldpc_decoder_cfg_t *decoder_cfg, void **plan);

/* Decode the planned batch: d_llr int16 arena, d_bits uint8 arena,
 * d_status / d_iterations int32 [num_blocks] (nullable).  With use_graph != 0
 * and a non-default stream, the launch (work-queue reset + kernel) is
 * captured once into a CUDA graph and replayed; it is re-captured when the
 * pointers, stream or tuning change.  Stream-ordered. */
int32_t nrldpc_mixed_plan_execute(void *plan, const int16_t *d_llr, uint8_t *d_bits,
                                  int32_t *d_status, int32_t *d_iterations,
                                  int32_t use_graph, void *stream);

/* Time the plan's candidates on the given data, keep the fastest and return
 * its index; ms_out (nullable) receives NRLDPC_MIXED_AUTOTUNE_CANDIDATES mean
 * times in ms.  Candidate k: code blocks per CTA (k < 4: each lifting size in
 * the CTA class that keeps more lifted rows active, 384-thread CTAs or
 * 256-thread CTAs with at most 240 active, three per SM; k >= 4: every size in
 * 384-thread CTAs) x CTAs per SM of the 384-thread class (2 for even k, 1 for
 * odd) x work order (largest items first for k mod 4 < 2, graphs interleaved
 * otherwise).  Synchronises the stream. */
#define NRLDPC_MIXED_AUTOTUNE_CANDIDATES 8
int32_t nrldpc_mixed_plan_autotune(void *plan, const int16_t *d_llr, uint8_t *d_bits,
                                   int32_t *d_status, int32_t *d_iterations,
                                   float *ms_out, void *stream);

/* Select autotuner candidate `candidate` (0 .. NRLDPC_MIXED_AUTOTUNE_CANDIDATES-1,
 * the same numbering) without timing anything.  A new plan starts at
 * candidate 0.  Returns 0, -4 for an unknown candidate, -1 on a CUDA error. */
int32_t nrldpc_mixed_plan_select(void *plan, int32_t candidate);

int32_t nrldpc_mixed_plan_destroy(void *plan);

/* ---- transport blocks: segmentation, batched decode, serving loop (no
 * counterpart in the reference's C ABI, which decodes single code blocks; the
 * segmentation formulas are TS 38.212 5.2.2 / 5.4.2.1 as restated in
 * py5gphy/ldpc/ldpc_info.py:59-109 and py5gphy/ldpc/nr_ldpc_ratematch.py:22-45) */

#define NRLDPC_TB_DROPPED (-5)   /* serving: not admitted (HBM budget exhausted) */
#define NRLDPC_TB_EXPIRED (-6)   /* serving: admitted, but waited longer than max_wait_s for a batch */

/* One transport block: A payload bits (multiple of 8), coded into G bits
 * (multiple of Qm, one layer) on base graph bgn.  Its G int16 LLRs start at
 * llr_offset in the LLR arena, code block after code block in order; its A/8
 * decoded payload bytes go to out_offset in the output arena.
 * tbs_lbrm > 0 selects limited-buffer rate matching (TS 38.212 5.4.2.1): each
 * code block's circular buffer holds Ncb = min(N, floor(3 tbs_lbrm / (2 C)))
 * bits (the reference always uses Ncb = N).
 * HARQ: with a soft-buffer arena passed to the decode call, code block r of
 * this block keeps its soft buffer (N + 2 Zc int16) at harq_offset +
 * r (N + 2 Zc); flags NRLDPC_TB_HARQ_COMBINE adds the received LLRs to the
 * stored soft buffer (retransmission with any rv), NRLDPC_TB_HARQ_STORE writes
 * the combined soft buffer back. */
#define NRLDPC_TB_HARQ_COMBINE 1
#define NRLDPC_TB_HARQ_STORE 2
typedef struct {
    int32_t A;
    int32_t G;
    uint16_t Qm;
    uint16_t rv;
    uint16_t bgn;
    uint16_t flags;
    int64_t llr_offset;
    int64_t out_offset;
    int32_t tbs_lbrm;
    int32_t pad;
    int64_t harq_offset;
} nrldpc_tb_t;

/* Segmentation of one transport block (host). */
typedef struct {
    int32_t C;          /* code blocks */
    int32_t L_tb;       /* transport-block CRC bits (16 or 24) */
    int32_t Kp;         /* K': information + code-block CRC bits per code block */
    int32_t Zc;
    int32_t E_lo, E_hi; /* code blocks 0..n_lo-1 carry E_lo coded bits, the rest E_hi */
    int32_t n_lo;
    ldpc_in_config_t cb_cfg;   /* per-code-block decoder configuration (E = E_lo) */
    int32_t Ncb;        /* circular-buffer length of every code block */
    int32_t k0;         /* start position of the block's rv in the circular buffer */
    int64_t harq_elems; /* int16 soft-buffer elements of the whole block: C (N + 2 Zc) */
} nrldpc_tb_info_t;

/* Returns 0, or NRLDPC_ERR_CONFIG with a reason on stderr: bad A / G / Qm /
 * bgn / rv, sizes that do not split into equal byte-aligned code blocks
 * (TS 38.214 transport-block sizes always do), or a code block whose E does
 * not fit 16 bits. */
int32_t nrldpc_tb_segment(const nrldpc_tb_t *tb, nrldpc_tb_info_t *info);

/* Base graph by TS 38.212 7.2.2 from A and the target code rate R (x 1024). */
int32_t nrldpc_tb_select_bg(int32_t A, int32_t R_x1024);

/* A decode engine for batches of up to max_tbs transport blocks and max_cbs
 * code blocks, with one fixed-point decoder setting (algos 1-3).  Each batch
 * is segmented on the device, all its code blocks decode in one persistent
 * launch (mixed sizes, CRC early exit per code block), and the transport-block
 * CRC and payload gather run on the device. */
int32_t nrldpc_tb_engine_create(int32_t max_tbs, int32_t max_cbs, const ldpc_decoder_cfg_t *decoder_cfg,
                                void **engine);
int32_t nrldpc_tb_engine_destroy(void *engine);

/* Decode num_tbs transport blocks described by d_tbs (device memory) whose LLRs
 * are in d_llr.  Writes the payload bytes of every block to d_out, d_status
 * [num_tbs] (0 CRC pass, 1 fail, -2 bad configuration, -4 batch over the
 * engine's capacity) and d_iterations [num_tbs] (largest code-block iteration
 * count; nullable).  d_harq (nullable) is the int16 soft-buffer arena the
 * blocks' HARQ flags and offsets refer to.  Stream-ordered, no host
 * synchronisation. */
int32_t nrldpc_tb_engine_decode(void *engine, const nrldpc_tb_t *d_tbs, int32_t num_tbs, const int16_t *d_llr,
                                uint8_t *d_out, int32_t *d_status, int32_t *d_iterations, int16_t *d_harq,
                                void *stream);

/* Device views of the last batch's code blocks, for inspection: hard bits
 * [max_cbs][1056] bytes, status and iterations [max_cbs], and each transport
 * block's first code-block index [max_tbs].  Any pointer may be NULL. */
int32_t nrldpc_tb_engine_views(void *engine, const uint8_t **d_cb_bits, const int32_t **d_cb_status,
                               const int32_t **d_cb_iterations, const int32_t **d_tb_first_cb);

/* Serving loop. */
typedef struct {
    int32_t max_batch_tbs;      /* transport blocks per decode batch at most */
    int32_t max_batch_cbs;      /* code blocks per decode batch at most */
    int64_t llr_budget_bytes;   /* HBM for the LLRs of admitted, unfinished blocks */
    int32_t pipeline_depth;     /* batches in flight, 1..16 (one engine lane each: ~90 MB of scratch) */
    int32_t pad;
    double timeout_s;           /* the run fails with NRLDPC_ERR_CUDA after this long */
    double max_wait_s;          /* > 0: an admitted block that has waited longer than this for a
                                   batch is dropped (NRLDPC_TB_EXPIRED), which bounds the queueing
                                   part of the latency past saturation; 0: no bound */
    /* Optional record of every decoded code block (all NULL: none).  Block i's
     * C code blocks go to indices h_cb_first[i] .. + C of the device arrays:
     * hard bits [..][1056] bytes, status and iterations.  Costs a device copy
     * per transport block: a checking aid, not for production. */
    const int64_t *h_cb_first;
    uint8_t *d_cb_bits;
    int32_t *d_cb_status;
    int32_t *d_cb_iterations;
} nrldpc_serve_cfg_t;

typedef struct {
    int64_t admitted, dropped, completed, failed, batches;
    double wall_s;              /* first arrival to last verdict */
    double mean_batch_tbs;
    int64_t expired;            /* admitted blocks dropped after max_wait_s */
} nrldpc_serve_stats_t;

/* Run the arrival trace tbs[i] / arrival_s[i] (host arrays, arrival times in
 * seconds from the start of the call, ascending) through the engine with
 * continuous batching: a block is admitted on arrival if its LLR bytes fit the
 * budget (else dropped: status NRLDPC_TB_DROPPED), admitted blocks form a new
 * batch whenever fewer than pipeline_depth batches are in flight (an admitted
 * block that waits longer than max_wait_s, when set, is dropped:
 * NRLDPC_TB_EXPIRED), and each block's verdict time is taken when its batch's
 * completion event is observed.
 * Writes h_status [n] and h_latency_s [n] (verdict - arrival; NaN if dropped).
 * All waits are host polls bounded by timeout_s; no device-side waits. */
int32_t nrldpc_serve_run(void *engine, const nrldpc_serve_cfg_t *cfg, const nrldpc_tb_t *tbs,
                         const double *arrival_s, int32_t n, const int16_t *d_llr, uint8_t *d_out,
                         int32_t *h_status, double *h_latency_s, nrldpc_serve_stats_t *stats, void *stream);

/* ---- differentiable unrolled float min-sum (no counterpart in the reference's
 * C ABI; the training model it serves is deep_learning/deeplearning_ldpc_model.py) */

/* Forward of `iterations` unrolled layered float min-sum iterations on batch
 * decoder-layout LLRs d_llr float [batch][N+2Zc], with per-(iteration, row)
 * d_alpha / d_beta float [iterations][rows], optional clip (<= 0: none).
 * Writes d_final [batch][N+2Zc], optionally every iteration's LLRs d_iter
 * [iterations][batch][N+2Zc], and the checkpoints the backward needs:
 * d_ck_lq float [iterations][batch][N+2Zc] and d_ck_lr uint32
 * [iterations][batch][rows][4 Zc] (per lifted row block: two magnitudes, the
 * sign-flip bits and the first-minimum index of every check row; sizes from
 * nrldpc_train_checkpoint_words).  No early termination.
 * Forward semantics: CTableNeuralLayeredMinSumDecoder.forward,
 * deep_learning/deeplearning_ldpc_model.py:315-410. */
int32_t nrldpc_train_forward(const float *d_llr, int32_t batch, const ldpc_in_config_t *cfg,
                             int32_t iterations, const float *d_alpha, const float *d_beta,
                             float clip, float *d_final, float *d_iter, float *d_ck_lq,
                             uint32_t *d_ck_lr, void *stream);

/* Backward of nrldpc_train_forward from its checkpoints: given the gradients
 * of the final LLRs (d_g_final, nullable) and of every iteration's LLRs
 * (d_g_iter, nullable), writes d_g_llr [batch][N+2Zc] and ADDS into d_g_alpha /
 * d_g_beta [iterations][rows].  detach != 0 stops gradients through the check
 * update inputs (the model's detach_check_update_inputs).  d_g_llr also holds
 * each block's running gradient between iterations, so it must not overlap
 * d_llr, d_g_iter or the checkpoints (it may be d_g_final itself). */
int32_t nrldpc_train_backward(const float *d_llr, int32_t batch, const ldpc_in_config_t *cfg,
                              int32_t iterations, const float *d_alpha, const float *d_beta,
                              float clip, int32_t detach, const float *d_ck_lq,
                              const uint32_t *d_ck_lr, const float *d_g_final,
                              const float *d_g_iter, float *d_g_llr, float *d_g_alpha,
                              float *d_g_beta, void *stream);

/* The same two kernels in float64, for gradient checks against finite
 * differences (float64 needs (N+2Zc) doubles of shared memory per code block:
 * BG1 Zc = 384 still fits).  d_ck_lr is then [iterations][batch][rows][6 Zc]
 * uint32 words. */
int32_t nrldpc_train_forward_f64(const double *d_llr, int32_t batch, const ldpc_in_config_t *cfg,
                                 int32_t iterations, const double *d_alpha, const double *d_beta,
                                 double clip, double *d_final, double *d_iter, double *d_ck_lq,
                                 uint32_t *d_ck_lr, void *stream);
int32_t nrldpc_train_backward_f64(const double *d_llr, int32_t batch, const ldpc_in_config_t *cfg,
                                  int32_t iterations, const double *d_alpha, const double *d_beta,
                                  double clip, int32_t detach, const double *d_ck_lq,
                                  const uint32_t *d_ck_lr, const double *d_g_final,
                                  const double *d_g_iter, double *d_g_llr, double *d_g_alpha,
                                  double *d_g_beta, void *stream);

/* Checkpoint sizes of one training forward: *lq_elems reals for d_ck_lq and
 * *msg_words uint32 words for d_ck_lr (f64 != 0: the float64 variant). */
int32_t nrldpc_train_checkpoint_words(const ldpc_in_config_t *cfg, int32_t iterations,
                                      int32_t batch, int32_t f64, int64_t *lq_elems,
                                      int64_t *msg_words);

/* Replace the per-(iteration, row) alpha/beta tables used by algo 2 for one
 * base graph (the reference compiles these in:
 * c_lib/BG1_trained_ldpc_weights.c:34,171, c_lib/BG2_trained_ldpc_weights.c).
 * alpha/beta are [num_iterations][rows] int16 Q15 / LLR units.  Iterations at
 * or beyond num_iterations reuse the last table row.  Passing NULL alpha
 * restores the built-in table.  Not safe to call while a decode is running. */
int32_t nrldpc_set_trained_weights(uint16_t bgn, const int16_t *alpha,
                                   const int16_t *beta, int32_t num_iterations);

/* Replace the 19-entry degree->alpha table used by algo 3 (entry d-1 is the
 * alpha of a degree-d row), as the reference's
 * layered_degree_minsum_ldpc_decode_with_alpha
 * (c_lib/degree_fixedpoint_ldpc_decoder.c:200-268) takes it per call.
 * NULL restores the default table. */
int32_t nrldpc_set_degree_alpha(const int16_t *degree_alpha);

/* Number of CUDA kernels this library has launched in this process. */
int64_t nrldpc_kernel_launch_count(void);

/* Library version string. */
const char *nrldpc_version(void);

/* No counterpart in the reference (its only checks are return codes).  Status
 * of the device-side index checks of the debug build
 * (libnrldpc_b200_debug.so, compiled with -DNRLDPC_BOUNDS_CHECK), which checks
 * every gather and scatter index of the decode kernels and records the first
 * violation instead of trapping: out[4] = {kind, index, limit, CTA} of that
 * violation (kind 1 belief word, 2 edge entry, 3 message scratch, 4 LLR
 * index, 5 CRC table entry; all zero when none), cleared when reset != 0.
 * Returns 1 in the debug build, 0 in the release build (out all zero). */
int32_t nrldpc_bounds_check_status(uint32_t *out, int32_t reset);

#ifdef __cplusplus
}
#endif

#endif /* NRLDPC_B200_H */
