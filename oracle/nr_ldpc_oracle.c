/*
 * nr_ldpc_oracle.c — CPU oracle (test infrastructure only; see the header).
 *
 * Plain-C restatement of the reference C library's receive path, written
 * from the reference's behaviour.  Each function cites the reference
 * file:line it restates.  Base-graph data comes from the 3GPP TS 38.212
 * tables generated into the package (nr_base_graphs.inc); the tables are
 * cross-checked against the reference library in tests/test_oracle_ref.py.
 */
#include "nr_ldpc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define BG1_ROWS 46
#define BG1_COLS 68
#define BG1_NNZ 316
#define BG2_ROWS 42
#define BG2_COLS 52
#define BG2_NNZ 197
#define MAX_DEG 19
#define MAX_ZC 384
#define LQ_MAX (BG1_COLS * MAX_ZC)
#define LR_MAX (BG1_NNZ * MAX_ZC)

typedef struct {
    uint8_t row, col;
    uint16_t v[8];
} nr_bg_edge_t;

#include "../deeplearning_5g_ldpc_decoder_b200/csrc/nr_base_graphs.inc"

typedef struct {
    int rows, cols, nnz;
    int off[BG1_ROWS + 1];
    int col[BG1_NNZ];
    int v[8][BG1_NNZ];
} graph_t;

static graph_t g_graph[2];
static int g_graph_ready = 0;

static void build(graph_t *g, const nr_bg_edge_t *e, int nnz, int rows, int cols) {
    g->rows = rows;
    g->cols = cols;
    g->nnz = nnz;
    int r = 0;
    g->off[0] = 0;
    for (int i = 0; i < nnz; i++) {
        while (e[i].row != r) g->off[++r] = i;
        g->col[i] = e[i].col;
        for (int s = 0; s < 8; s++) g->v[s][i] = e[i].v[s];
    }
    while (r < rows) g->off[++r] = nnz;
}

static const graph_t *graph(int bgn) {
    if (!g_graph_ready) {
        build(&g_graph[0], kBG1Edges, BG1_NNZ, BG1_ROWS, BG1_COLS);
        build(&g_graph[1], kBG2Edges, BG2_NNZ, BG2_ROWS, BG2_COLS);
        g_graph_ready = 1;
    }
    return &g_graph[bgn == 1 ? 0 : 1];
}

int orc_graph(const orc_params_t *p, int32_t *col, int32_t *shift, int32_t *off) {
    if (!p || (p->bgn != 1 && p->bgn != 2) || p->Zc <= 0) return -1;
    const graph_t *g = graph(p->bgn);
    for (int i = 0; i < g->nnz; i++) {
        col[i] = g->col[i];
        shift[i] = g->v[p->iLS][i] % p->Zc;
    }
    for (int r = 0; r <= g->rows; r++) off[r] = g->off[r];
    return g->nnz;
}

/* ------------------------------------------------------------ parameters */
/* c_lib/ldpc_internal.c:13-22 (TS 38.212 Table 5.3.2-1) and :24-64. */
static const int kSets[8][8] = {
    {2, 4, 8, 16, 32, 64, 128, 256}, {3, 6, 12, 24, 48, 96, 192, 384}, {5, 10, 20, 40, 80, 160, 320, 0},
    {7, 14, 28, 56, 112, 224, 0, 0}, {9, 18, 36, 72, 144, 288, 0, 0},  {11, 22, 44, 88, 176, 352, 0, 0},
    {13, 26, 52, 104, 208, 0, 0, 0}, {15, 30, 60, 120, 240, 0, 0, 0}};

int orc_derive(const orc_in_config_t *in, orc_params_t *p) {
    memset(p, 0, sizeof(*p));
    p->bgn = in->bgn;
    p->A = in->A;
    p->crctype = in->crctype;
    p->E = in->E;
    p->rv = in->rv;
    p->Qm = in->Qm;
    p->HARQ_on = in->HARQ_on;
    /* validation order of c_lib/ldpc_internal.c:84-123 */
    if (in->bgn != 1 && in->bgn != 2) return -1;
    if (in->crctype > 3) return -1;
    if (in->Qm != 1 && in->Qm != 2 && in->Qm != 4 && in->Qm != 6 && in->Qm != 8) return -1;
    if (in->HARQ_on != 0 && in->HARQ_on != 1) return -1;
    if (in->rv > 3) return -1;
    if (in->E % in->Qm != 0) return -1;
    if (in->A % 8 != 0) return -1;
    p->B = (uint16_t)(in->A + (in->crctype == 0 ? 16 : 24)); /* uint16_t field */
    if (in->bgn == 1 && p->B > 8448) return -1;
    if (in->bgn == 2 && p->B > 3840) return -1;
    int Kb;
    if (in->bgn == 1) Kb = 22;
    else if (p->B > 640) Kb = 10;
    else if (p->B > 560) Kb = 9;
    else if (p->B > 192) Kb = 8;
    else Kb = 6;
    int best = 65535, set = -1;
    for (int s = 0; s < 8; s++)
        for (int j = 0; j < 8 && kSets[s][j]; j++)
            if (Kb * kSets[s][j] >= p->B) {
                if (kSets[s][j] < best) { best = kSets[s][j]; set = s; }
                break;
            }
    p->Zc = best;
    p->iLS = set;
    p->K = (in->bgn == 1 ? 22 : 10) * p->Zc;
    p->N = (in->bgn == 1 ? 66 : 50) * p->Zc;
    p->F = p->K - p->B;
    static const int k0a[4] = {0, 17, 33, 56}, k0b[4] = {0, 13, 25, 43};
    p->k0 = (in->bgn == 1 ? k0a : k0b)[in->rv] * p->Zc;
    p->Ncb = p->N;
    const graph_t *g = graph(in->bgn);
    p->rows = g->rows;
    p->cols = g->cols;
    p->nnz = g->nnz;
    return 0;
}

int orc_set_ncb(orc_params_t *p, int ncb) {
    if (ncb <= 0 || ncb >= p->N) {
        p->Ncb = p->N;
        return 0;
    }
    if (ncb < p->K - 2 * p->Zc) return -1;
    static const int fa[4] = {0, 17, 33, 56}, fb[4] = {0, 13, 25, 43};
    const int f = (p->bgn == 1 ? fa : fb)[p->rv];
    const int nbg = p->bgn == 1 ? 66 : 50;
    p->Ncb = ncb;
    p->k0 = (int)(((long long)f * ncb) / ((long long)nbg * p->Zc)) * p->Zc;
    return 0;
}

/* ------------------------------------------------------------------ CRC */
/* c_lib/nr_crc.c:93-140: MSB-first byte table, remainder of M(x)*x^W. */
uint32_t orc_crc(const uint8_t *data, int len, int crctype) {
    int width;
    uint32_t poly;
    switch (crctype) {
        case 0: width = 16; poly = 0x1021; break;
        case 1: width = 24; poly = 0x864CFB; break;
        case 2: width = 24; poly = 0x800063; break;
        case 3: width = 24; poly = 0xB2B117; break;
        default: return 0;
    }
    const uint32_t mask = (1u << width) - 1u, top = 1u << (width - 1);
    uint32_t crc = 0;
    for (int i = 0; i < len; i++) {
        crc ^= (uint32_t)data[i] << (width - 8);
        for (int b = 0; b < 8; b++) crc = (crc & top) ? ((crc << 1) ^ poly) : (crc << 1);
        crc &= mask;
    }
    return crc & mask;
}

/* -------------------------------------------------------- rate recovery */
/* c_lib/ldpc_rate_recovery.c:24-65, the same sequential walk. */
void orc_rate_recover(const orc_params_t *p, int16_t fill, const int16_t *llr, int16_t *harq) {
    const int E = p->E, N = p->N, Zc = p->Zc, Qm = p->Qm;
    const int symbols = Qm ? E / Qm : 0;
    if (p->HARQ_on == 0) memset(harq, 0, sizeof(int16_t) * (N + 2 * Zc));
    for (int i = 0; i < p->F; i++) harq[p->B + i] = fill;
    int k = 0, pos = p->k0;
    while (k < E) {
        const int bit = k / symbols, sym = k % symbols;
        const int idx = sym * Qm + bit;
        if (pos < p->B - 2 * Zc || pos >= p->K - 2 * Zc) {
            harq[pos + 2 * Zc] = (int16_t)(harq[pos + 2 * Zc] + llr[idx]);
            k++;
        }
        pos = (pos + 1) % p->Ncb;
    }
}

/* --------------------------------------------------- algo-2 / 3 tables */
static int16_t *g_tr_alpha[2], *g_tr_beta[2];
static int g_tr_T[2];
static int16_t g_deg_alpha[MAX_DEG];
static int g_deg_ready = 0;

static int16_t default_degree_alpha(int d) { return d <= 4 ? 26623 : (d <= 8 ? 24575 : 22527); }

void orc_set_trained(int bgn, const int16_t *alpha, const int16_t *beta, int T) {
    const int k = bgn == 1 ? 0 : 1;
    const graph_t *g = graph(bgn);
    free(g_tr_alpha[k]);
    free(g_tr_beta[k]);
    if (!alpha) T = 32;
    g_tr_T[k] = T;
    g_tr_alpha[k] = (int16_t *)malloc(sizeof(int16_t) * T * g->rows);
    g_tr_beta[k] = (int16_t *)malloc(sizeof(int16_t) * T * g->rows);
    for (int it = 0; it < T; it++)
        for (int r = 0; r < g->rows; r++) {
            const int i = it * g->rows + r;
            if (alpha) {
                g_tr_alpha[k][i] = alpha[i];
                g_tr_beta[k][i] = beta ? beta[i] : 0;
            } else {
                /* built-in table: degree rule for every iteration, beta 0
                 * (c_lib/BG1_trained_ldpc_weights.c:25-33) */
                g_tr_alpha[k][i] = default_degree_alpha(g->off[r + 1] - g->off[r]);
                g_tr_beta[k][i] = 0;
            }
        }
}

void orc_set_degree_alpha(const int16_t *tab) {
    for (int d = 0; d < MAX_DEG; d++) g_deg_alpha[d] = tab ? tab[d] : default_degree_alpha(d + 1);
    g_deg_ready = 1;
}

/* ------------------------------------------------- fixed-point decoders */
static int16_t LQ[LQ_MAX];
static int16_t LR[LR_MAX];
static float LQF[LQ_MAX];
static float LRF[LR_MAX];

static void pack_bits_i16(const int16_t *lq, uint8_t *bits, int B) {
    for (int i = 0; i < B; i++) bits[i / 8] = (uint8_t)((bits[i / 8] << 1) | (lq[i] < 0 ? 1 : 0));
}

static void pack_bits_f32(const float *lq, uint8_t *bits, int B) {
    for (int i = 0; i < B; i++) bits[i / 8] = (uint8_t)((bits[i / 8] << 1) | (lq[i] < 0.0f ? 1 : 0));
}

/* One lifted check-node update, c_lib/fixedpoint_ldpc_decoder.c:103-144. */
static void cn_update_fixed(int deg, const int *cols, int16_t *lr, int16_t alpha, int16_t beta, int16_t mx,
                            int16_t mn) {
    int16_t rel[MAX_DEG];
    int sign = 1;
    int m1 = 32767, m2 = 32767, idx = -1;
    for (int j = 0; j < deg; j++) {
        rel[j] = (int16_t)(LQ[cols[j]] - lr[j]);              /* int16 wrap, :203 */
        int a = rel[j];
        if (a < 0) {
            sign = -sign;
            a = (a == -32768) ? 32767 : -a;                   /* :48-55 */
        }
        if (a < m1) { m2 = m1; m1 = a; idx = j; }             /* :57-66 */
        else if (a < m2) m2 = a;
    }
    if (m1 > mx) m1 = mx;                                     /* :121-122 */
    if (m2 > mx) m2 = mx;
    int o1 = m1 - beta, o2 = m2 - beta;                       /* :38-46 */
    if (o1 < 0) o1 = 0;
    if (o2 < 0) o2 = 0;
    const int16_t n1 = (int16_t)((alpha * o1 + (1 << 14)) >> 15);
    const int16_t n2 = (int16_t)((alpha * o2 + (1 << 14)) >> 15);
    for (int j = 0; j < deg; j++) {
        const int16_t v = (j == idx) ? n2 : n1;
        lr[j] = (int16_t)(rel[j] >= 0 ? sign * v : -sign * v);
        const int32_t s = (int32_t)rel[j] + (int32_t)lr[j];
        LQ[cols[j]] = (int16_t)(s > mx ? mx : (s < mn ? mn : s)); /* :28-36 */
    }
}

/* Layered schedule, c_lib/fixedpoint_ldpc_decoder.c:162-222, with alpha/beta
 * per (iteration, row) chosen by algo (1: config; 2: trained table,
 * c_lib/neural_fixedpoint_ldpc_decoder.c:248-250; 3: degree table,
 * c_lib/degree_fixedpoint_ldpc_decoder.c:244-259). */
static int32_t decode_fixed(const int16_t *harq, uint8_t *bits, const orc_params_t *p, const orc_decoder_cfg_t *c,
                            int16_t *lq_out, int32_t *iters) {
    const graph_t *g = graph(p->bgn);
    const int Zc = p->Zc;
    const int k = p->bgn == 1 ? 0 : 1;
    if (c->algo == 2 && !g_tr_alpha[k]) orc_set_trained(p->bgn, NULL, NULL, 0);
    if (c->algo == 3 && !g_deg_ready) orc_set_degree_alpha(NULL);
    memcpy(LQ, harq, sizeof(int16_t) * (p->N + 2 * Zc));
    memset(LR, 0, sizeof(int16_t) * g->nnz * Zc);
    int32_t ret = 1, it;
    for (it = 0; it < c->max_iterations; it++) {
        for (int r = 0; r < g->rows; r++) {
            const int off = g->off[r], deg = g->off[r + 1] - off;
            int16_t alpha = (int16_t)c->alpha, beta = (int16_t)c->beta;
            if (c->algo == 2) {
                const int t = it < g_tr_T[k] ? it : g_tr_T[k] - 1;
                alpha = g_tr_alpha[k][t * g->rows + r];
                beta = g_tr_beta[k][t * g->rows + r];
            } else if (c->algo == 3) {
                alpha = g_deg_alpha[deg > MAX_DEG ? MAX_DEG - 1 : (deg == 0 ? 0 : deg - 1)];
            }
            for (int zx = 0; zx < Zc; zx++) {
                int cols[MAX_DEG];
                for (int j = 0; j < deg; j++) cols[j] = g->col[off + j] * Zc + (g->v[p->iLS][off + j] + zx) % Zc;
                cn_update_fixed(deg, cols, LR + off * Zc + zx * deg, alpha, beta, c->max_llr, c->min_llr);
            }
        }
        pack_bits_i16(LQ, bits, p->B);
        if (orc_crc(bits, p->B / 8, p->crctype) == 0) {
            ret = 0;
            it++;
            break;
        }
    }
    if (iters) *iters = it;
    if (lq_out) memcpy(lq_out, LQ, sizeof(int16_t) * (p->N + 2 * Zc));
    return ret;
}

/* ------------------------------------------------------ float min-sum */
/* c_lib/floatpoint_ldpc_decoder.c:189-220 and :307-366. */
static float clipf(float v, float mx, float mn) { return v > mx ? mx : (v < mn ? mn : v); }

static void cn_update_fms(int deg, const int *cols, float *lr, float alpha, float beta, float mx, float mn) {
    float rel[MAX_DEG];
    float m1 = FLT_MAX, m2 = FLT_MAX;
    int idx = 0, sign = 1;
    for (int j = 0; j < deg; j++) {
        rel[j] = LQF[cols[j]] - lr[j];
        if (rel[j] < 0.0f) sign = -sign;
        const float a = fabsf(rel[j]);
        if (a < m1) { m2 = m1; m1 = a; idx = j; }
        else if (a < m2) m2 = a;
    }
    m1 = clipf(m1, mx, 0.0f);
    m2 = clipf(m2, mx, 0.0f);
    float o1 = m1 - beta, o2 = m2 - beta;
    if (o1 < 0.0f) o1 = 0.0f;
    if (o2 < 0.0f) o2 = 0.0f;
    const float n1 = alpha * o1, n2 = alpha * o2;
    for (int j = 0; j < deg; j++) {
        const float v = (j == idx) ? n2 : n1;
        const float es = (rel[j] < 0.0f) ? -(float)sign : (float)sign;
        lr[j] = es * v;
        LQF[cols[j]] = clipf(rel[j] + lr[j], mx, mn);
    }
}

/* ----------------------------------------------------------------- BP */
/* c_lib/floatpoint_ldpc_decoder.c:53-151 and :237-298. */
static float bp_msg(float prod) {
    if (prod >= 1.0f) return 2.0f * 19.07f;
    if (prod <= -1.0f) return -2.0f * 19.07f;
    return 2.0f * atanhf(prod);
}

static void cn_update_bp(int deg, const int *cols, float *lr) {
    float rel[MAX_DEG], th[MAX_DEG];
    int nz = 0, zidx = -1;
    float prod = 1.0f;
    for (int j = 0; j < deg; j++) {
        rel[j] = LQF[cols[j]] - lr[j];
        if (rel[j] == 0.0f) {
            nz++;
            zidx = j;
            th[j] = 0.0f;
        } else {
            th[j] = tanhf(rel[j] / 2.0f);
            prod *= th[j];
        }
    }
    if (nz == 1) {
        for (int j = 0; j < deg; j++) lr[j] = 0.0f;
        lr[zidx] = bp_msg(prod);
    } else if (nz >= 2) {
        for (int j = 0; j < deg; j++) lr[j] = 0.0f;
    } else {
        float pre[MAX_DEG + 1], suf[MAX_DEG + 1];
        pre[0] = 1.0f;
        for (int j = 0; j < deg; j++) pre[j + 1] = pre[j] * th[j];
        suf[deg] = 1.0f;
        for (int j = deg - 1; j >= 0; j--) suf[j] = suf[j + 1] * th[j];
        for (int j = 0; j < deg; j++) lr[j] = bp_msg(pre[j] * suf[j + 1]);
    }
    for (int j = 0; j < deg; j++) LQF[cols[j]] = rel[j] + lr[j];
}

static int32_t decode_float(const int16_t *harq, uint8_t *bits, const orc_params_t *p, const orc_decoder_cfg_t *c,
                            float *lq_out, int32_t *iters) {
    const graph_t *g = graph(p->bgn);
    const int Zc = p->Zc;
    const int bp = c->algo == 0;
    const float alpha = (float)c->alpha / 32768.0f, beta = (float)c->beta / 128.0f;
    const float mx = (float)c->max_llr / 128.0f, mn = (float)c->min_llr / 128.0f;
    for (int i = 0; i < p->N + 2 * Zc; i++) LQF[i] = (float)harq[i] / 128.0f;
    for (int i = 0; i < g->nnz * Zc; i++) LRF[i] = 0.0f;
    int32_t ret = 1, it;
    for (it = 0; it < c->max_iterations; it++) {
        for (int r = 0; r < g->rows; r++) {
            const int off = g->off[r], deg = g->off[r + 1] - off;
            for (int zx = 0; zx < Zc; zx++) {
                int cols[MAX_DEG];
                for (int j = 0; j < deg; j++) cols[j] = g->col[off + j] * Zc + (g->v[p->iLS][off + j] + zx) % Zc;
                float *lr = LRF + off * Zc + zx * deg;
                if (bp) cn_update_bp(deg, cols, lr);
                else cn_update_fms(deg, cols, lr, alpha, beta, mx, mn);
            }
        }
        pack_bits_f32(LQF, bits, p->B);
        if (orc_crc(bits, p->B / 8, p->crctype) == 0) {
            ret = 0;
            it++;
            break;
        }
    }
    if (iters) *iters = it;
    if (lq_out) memcpy(lq_out, LQF, sizeof(float) * (p->N + 2 * Zc));
    return ret;
}

int32_t orc_decode_recovered(const int16_t *harq, uint8_t *hardbits, const orc_params_t *p,
                             const orc_decoder_cfg_t *cfg, void *lq_out, int32_t *iters_out) {
    switch (cfg->algo) {
        case 1:
        case 2:
        case 3:
            return decode_fixed(harq, hardbits, p, cfg, (int16_t *)lq_out, iters_out);
        case 0:
        case 4:
            return decode_float(harq, hardbits, p, cfg, (float *)lq_out, iters_out);
        default:
            return -3;
    }
}

int32_t orc_decode(const int16_t *llr, uint8_t *hardbits, const orc_in_config_t *in, const orc_decoder_cfg_t *cfg,
                   int16_t *harq, void *lq_out, int32_t *iters_out) {
    orc_params_t p;
    if (orc_derive(in, &p) != 0) return -2;
    orc_rate_recover(&p, cfg->filling_bit_value, llr, harq);
    return orc_decode_recovered(harq, hardbits, &p, cfg, lq_out, iters_out);
}

int32_t orc_decode_many(const int16_t *llr, int64_t llr_stride, int32_t n, const orc_in_config_t *in,
                        const orc_decoder_cfg_t *cfg, uint8_t *bits, int64_t bits_stride, int32_t *status,
                        int32_t *iters) {
    static int16_t harq[LQ_MAX];
    orc_in_config_t fresh = *in;
    fresh.HARQ_on = 0;
    orc_params_t p;
    if (orc_derive(&fresh, &p) != 0) return -2;
    for (int32_t i = 0; i < n; i++) {
        uint8_t *b = bits + (int64_t)i * bits_stride;
        memset(b, 0, (p.B + 7) / 8);
        int32_t it = 0;
        const int32_t rc = orc_decode(llr + (int64_t)i * llr_stride, b, &fresh, cfg, harq, NULL, &it);
        if (rc < 0) return rc;
        if (status) status[i] = rc;
        if (iters) iters[i] = it;
    }
    return 0;
}

/* -------------------------------------------------------------- encoder */
/* c_lib/ldpc_encoder.c:52-242: parity from the first four rows (double-
 * diagonal core) then the extension rows. */
static int encode_bits(const uint8_t *cbits, uint8_t *out, const orc_params_t *p) {
    const graph_t *g = graph(p->bgn);
    const int Zc = p->Zc, K = p->K, Kb = K / Zc;
    static uint8_t L[4][MAX_ZC], pc[4][MAX_ZC];
    memcpy(out, cbits, (size_t)K);
    for (int r = 0; r < 4; r++)
        for (int zx = 0; zx < Zc; zx++) {
            int s = 0;
            for (int e = g->off[r]; e < g->off[r + 1]; e++)
                if (g->col[e] < Kb) s += out[g->col[e] * Zc + (g->v[p->iLS][e] + zx) % Zc];
            L[r][zx] = (uint8_t)(s & 1);
        }
    int sh0, sh1;
    if (p->bgn == 1) {
        sh0 = g->v[p->iLS][g->off[0] + 17];
        sh1 = g->v[p->iLS][g->off[1] + 16];
    } else {
        sh0 = g->v[p->iLS][g->off[0] + 6];
        sh1 = g->v[p->iLS][g->off[2] + 5];
    }
    for (int zx = 0; zx < Zc; zx++) pc[0][(sh1 + zx) % Zc] = (uint8_t)(L[0][zx] ^ L[1][zx] ^ L[2][zx] ^ L[3][zx]);
    for (int zx = 0; zx < Zc; zx++) {
        const uint8_t t = pc[0][(sh0 + zx) % Zc];
        pc[1][zx] = L[0][zx] ^ t;
        pc[3][zx] = L[3][zx] ^ t;
    }
    for (int zx = 0; zx < Zc; zx++) pc[2][zx] = p->bgn == 1 ? (L[2][zx] ^ pc[3][zx]) : (L[1][zx] ^ pc[1][zx]);
    for (int q = 0; q < 4; q++)
        for (int zx = 0; zx < Zc; zx++) out[K + q * Zc + zx] = pc[q][zx];
    for (int r = 4; r < g->rows; r++)
        for (int zx = 0; zx < Zc; zx++) {
            int s = 0;
            for (int e = g->off[r]; e < g->off[r + 1]; e++)
                if (g->col[e] < Kb + 4) s += out[g->col[e] * Zc + (g->v[p->iLS][e] + zx) % Zc];
            out[K + r * Zc + zx] = (uint8_t)(s & 1);
        }
    return 0;
}

int32_t orc_encode_codeword(const uint8_t *infobytes, uint8_t *cw_bits, const orc_in_config_t *in) {
    orc_params_t p;
    if (orc_derive(in, &p) != 0) return -2;
    static uint8_t c[22 * MAX_ZC];
    const uint32_t crc = orc_crc(infobytes, p.A / 8, p.crctype);
    const int L = p.B - p.A;
    for (int i = 0; i < p.A; i++) c[i] = (infobytes[i / 8] >> (7 - i % 8)) & 1;
    for (int i = 0; i < L; i++) c[p.A + i] = (crc >> (L - 1 - i)) & 1;
    memset(c + p.B, 0, (size_t)p.F);
    return encode_bits(c, cw_bits, &p);
}

/* c_lib/ldpc_rate_match.c:27-106: bit selection from k0 over the circular
 * buffer without filler bits, then the Qm row/column interleave. */
int32_t orc_encode_params(const uint8_t *infobytes, uint8_t *rm_bytes, const orc_params_t *pp) {
    const orc_params_t p = *pp;
    static uint8_t cw[BG1_COLS * MAX_ZC];
    static uint8_t e[65536];
    orc_in_config_t in = {(uint16_t)p.bgn, (uint16_t)p.A, (uint16_t)p.crctype, (uint16_t)p.E,
                          (uint16_t)p.rv, (uint16_t)p.Qm, 0};
    orc_encode_codeword(infobytes, cw, &in);
    const int Zc = p.Zc;
    int k = 0, pos = p.k0;
    while (k < p.E) {
        if (pos < p.B - 2 * Zc || pos >= p.K - 2 * Zc) e[k++] = cw[pos + 2 * Zc];
        pos = (pos + 1) % p.Ncb;
    }
    const int sym = p.E / p.Qm;
    memset(rm_bytes, 0, (size_t)(p.E + 7) / 8);
    for (int t = 0; t < p.E; t++) {
        const int s = t / p.Qm, b = t % p.Qm;
        if (e[b * sym + s]) rm_bytes[t / 8] |= (uint8_t)(0x80 >> (t % 8));
    }
    return 0;
}

int32_t orc_encode(const uint8_t *infobytes, uint8_t *rm_bytes, const orc_in_config_t *in) {
    orc_params_t p;
    if (orc_derive(in, &p) != 0) return -2;
    return orc_encode_params(infobytes, rm_bytes, &p);
}

/* -------------------------------------------------------------- channel */
static uint64_t sm_next(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double uni(uint64_t *s) { return ((double)(sm_next(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

static double gauss(uint64_t *s) {
    const double u1 = uni(s), u2 = uni(s);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* One PAM dimension of NR QAM (TS 38.211 5.1): amplitude from m label bits,
 * the first bit giving the sign. */
static double pam_level(const int *bits, int m) {
    double a = 1.0;
    for (int i = m - 1; i >= 1; i--) a = (double)(1 << (m - i)) - (1 - 2 * bits[i]) * a;
    return (1 - 2 * bits[0]) * a;
}

static int16_t quantize(double llr) {
    const float s = (float)llr * 128.0f;
    int32_t q = (int32_t)(s >= 0.0f ? s + 0.5f : s - 0.5f);
    if (q > 10000) q = 10000;
    if (q < -10000) q = -10000;
    return (int16_t)q;
}

int orc_channel(const uint8_t *inbytes, size_t num_bits, uint16_t Qm, float noise_power_db, uint64_t seed,
                int16_t *llr_out) {
    if (!inbytes || !llr_out || num_bits == 0) return -1;
    if (Qm != 1 && Qm != 2 && Qm != 4 && Qm != 6 && Qm != 8) return -1;
    if (num_bits % Qm) return -1;
    const double nv = pow(10.0, noise_power_db / 10.0), sigma = sqrt(nv / 2.0);
    const int m = Qm == 1 ? 1 : Qm / 2;
    double norm;
    switch (Qm) {
        case 1: case 2: norm = sqrt(2.0); break;
        case 4: norm = sqrt(10.0); break;
        case 6: norm = sqrt(42.0); break;
        default: norm = sqrt(170.0); break;
    }
    const int L = 1 << m;
    double lev[16];
    int lab[16][4];
    for (int v = 0; v < L; v++) {
        for (int i = 0; i < m; i++) lab[v][i] = (v >> (m - 1 - i)) & 1;
        lev[v] = pam_level(lab[v], m) / norm;
    }
    uint64_t st = seed * 0x2545F4914F6CDD1Dull + 1;
    const size_t nsym = num_bits / Qm;
    for (size_t s = 0; s < nsym; s++) {
        int b[8];
        for (int j = 0; j < Qm; j++) {
            const size_t i = s * Qm + j;
            b[j] = (inbytes[i / 8] >> (7 - i % 8)) & 1;
        }
        double re, im;
        if (Qm == 1) {
            re = im = (1 - 2 * b[0]) / norm;
        } else {
            int br[4], bi[4];
            for (int i = 0; i < m; i++) {
                br[i] = b[2 * i];
                bi[i] = b[2 * i + 1];
            }
            re = pam_level(br, m) / norm;
            im = pam_level(bi, m) / norm;
        }
        re += sigma * gauss(&st);
        im += sigma * gauss(&st);
        if (Qm == 1) {
            const double A = 1.0 / norm;
            llr_out[s] = quantize(4.0 * (re + im) * A / nv);
            continue;
        }
        /* exact max-log LLR per dimension: (min d^2 | bit=1) - (min d^2 | bit=0) */
        for (int dim = 0; dim < 2; dim++) {
            const double y = dim == 0 ? re : im;
            for (int i = 0; i < m; i++) {
                double d0 = 1e300, d1 = 1e300;
                for (int v = 0; v < L; v++) {
                    const double d = (y - lev[v]) * (y - lev[v]);
                    if (lab[v][i]) { if (d < d1) d1 = d; }
                    else if (d < d0) d0 = d;
                }
                llr_out[s * Qm + 2 * i + dim] = quantize((d1 - d0) / nv);
            }
        }
    }
    return 0;
}
