/*
 * nr_ldpc_oracle.h — CPU oracle for the 5G NR LDPC receive path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * C library algorithms (hahaliu2001/deeplearning_5g_ldpc_decoder, c_lib/),
 * written to check the CUDA path.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks this oracle against
 * golden vectors produced by the reference C library itself
 * (tests/golden/make_golden.py), and, where the reference tree is present,
 * against the reference library built from source (oracle/build_ref.sh).
 */
#ifndef NR_LDPC_ORACLE_H
#define NR_LDPC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint16_t bgn, A, crctype, E, rv, Qm, HARQ_on;
} orc_in_config_t;

typedef struct {
    uint16_t algo, max_iterations, alpha, beta;
    int16_t filling_bit_value, max_llr, min_llr;
} orc_decoder_cfg_t;

typedef struct {
    int bgn, A, crctype, E, rv, Qm, HARQ_on;
    int B, Zc, iLS, K, F, N, k0;
    int rows, cols, nnz;
    int Ncb;   /* circular-buffer length: N, or less with limited-buffer rate matching */
} orc_params_t;

/* gen_ldpc_parameters (c_lib/ldpc_internal.c:66-170). 0 ok, -1 invalid. */
int orc_derive(const orc_in_config_t *in, orc_params_t *p);

/* Base-graph tables of one configuration in the reference's CSR layout
 * (ldpc_config_t of c_lib/nr_ldpc.h: HBG_array / Vij_array / HBG_offset_array):
 * col[nnz] base columns, shift[nnz] = Vij mod Zc for the configuration's
 * lifting set, off[rows+1] row offsets.  Returns nnz, or -1. */
int orc_graph(const orc_params_t *p, int32_t *col, int32_t *shift, int32_t *off);

/* Limited-buffer rate matching (TS 38.212 5.4.2.1): circular buffer of ncb
 * bits (0 < ncb < N; ncb >= K-2Zc so the systematic part is whole) and k0
 * recomputed for it.  The reference always uses Ncb = N; this is restated from
 * the standard as py5gphy/ldpc/nr_ldpc_ratematch.py:48-67 does.  0 ok, -1 bad. */
int orc_set_ncb(orc_params_t *p, int ncb);

/* Rate matching of one block with explicit parameters (Ncb honoured). */
int32_t orc_encode_params(const uint8_t *infobytes, uint8_t *rm_bytes, const orc_params_t *p);

/* calculate_crc (c_lib/nr_crc.c:170-179). */
uint32_t orc_crc(const uint8_t *data, int len, int crctype);

/* nr_ldpc_rate_recover_harq_combine (c_lib/ldpc_rate_recovery.c:24-65) into a
 * caller-owned soft buffer of at least N+2Zc int16. */
void orc_rate_recover(const orc_params_t *p, int16_t fill, const int16_t *llr, int16_t *harq);

/* Algo-2 tables: [T][rows] alpha / beta for one base graph; T iterations.
 * Iterations >= T reuse the last row.  NULL alpha restores the built-in
 * degree-rule table (32 iterations, beta 0). */
void orc_set_trained(int bgn, const int16_t *alpha, const int16_t *beta, int T);
/* Algo-3 degree table (19 entries) or NULL for the default. */
void orc_set_degree_alpha(const int16_t *tab);

/* Decode from a recovered soft buffer (N+2Zc int16).  hardbits gets
 * ceil(B/8) bytes (shift-accumulated like the reference: zero it first).
 * lq_out: final beliefs (int16 for algos 1-3, float for 0/4), N+2Zc values,
 * may be NULL.  iters_out: iterations executed, may be NULL.
 * Returns 0 CRC pass, 1 not converged, -3 bad algo. */
int32_t orc_decode_recovered(const int16_t *harq, uint8_t *hardbits, const orc_params_t *p,
                             const orc_decoder_cfg_t *cfg, void *lq_out, int32_t *iters_out);

/* c_ldpc_5g_decode (c_lib/c_ldpc_5g_decoder.c:34-79) with an explicit soft
 * buffer (68*384 int16) standing in for the reference's global one. */
int32_t orc_decode(const int16_t *llr, uint8_t *hardbits, const orc_in_config_t *in,
                   const orc_decoder_cfg_t *cfg, int16_t *harq, void *lq_out, int32_t *iters_out);

/* Decode n code blocks with one configuration (HARQ off), for timing. */
int32_t orc_decode_many(const int16_t *llr, int64_t llr_stride, int32_t n, const orc_in_config_t *in,
                        const orc_decoder_cfg_t *cfg, uint8_t *bits, int64_t bits_stride,
                        int32_t *status, int32_t *iters);

/* c_ldpc_5g_encode (c_lib/c_ldpc_5g_encoder.c:66-88): CRC attach, LDPC
 * encode (c_lib/ldpc_encoder.c:221-242), rate match + bit interleave
 * (c_lib/ldpc_rate_match.c:27-106).  rm_bytes gets ceil(E/8) bytes. */
int32_t orc_encode(const uint8_t *infobytes, uint8_t *rm_bytes, const orc_in_config_t *in);

/* Codeword bits (one per byte) of the full encoder output, N+2Zc long. */
int32_t orc_encode_codeword(const uint8_t *infobytes, uint8_t *cw_bits, const orc_in_config_t *in);

/* Test channel in the style of tx_rx_process (c_lib/tx_rx_process.c:286-324):
 * NR QAM mapping, complex AWGN of power 10^(noise_db/10), max-log LLRs,
 * round(128*llr) clipped to +-10000.  The noise comes from this oracle's own
 * seeded generator (splitmix64 + Box-Muller), not from libc rand(). */
int orc_channel(const uint8_t *inbytes, size_t num_bits, uint16_t Qm, float noise_power_db, uint64_t seed,
                int16_t *llr_out);

#ifdef __cplusplus
}
#endif

#endif
