// nrldpc_tables.cpp — base graphs, parameter derivation and host CRC.
//
// The arithmetic here is the host half of the drop-in boundary: it must give
// the same B, Zc, iLS, K, F, N and k0 as the reference's gen_ldpc_parameters
// (c_lib/ldpc_internal.c:66-170) and the same CRC remainders as its
// calculate_crc (c_lib/nr_crc.c:129-179).
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

struct nr_bg_edge_t {
  uint8_t row, col;
  uint16_t v[8];
};

#include "nr_base_graphs.inc"

// TS 38.212 Table 5.3.2-1: the 51 lifting sizes, grouped by set index iLS.
const uint16_t kLiftingSets[8][8] = {
    {2, 4, 8, 16, 32, 64, 128, 256}, {3, 6, 12, 24, 48, 96, 192, 384},
    {5, 10, 20, 40, 80, 160, 320, 0}, {7, 14, 28, 56, 112, 224, 0, 0},
    {9, 18, 36, 72, 144, 288, 0, 0},  {11, 22, 44, 88, 176, 352, 0, 0},
    {13, 26, 52, 104, 208, 0, 0, 0},  {15, 30, 60, 120, 240, 0, 0, 0},
};

BaseGraph g_bg[2];
std::once_flag g_bg_once;

void build_graph(BaseGraph* g, int bgn, const nr_bg_edge_t* e, int nnz, int rows, int cols) {
  memset(g, 0, sizeof(*g));
  g->bgn = bgn;
  g->rows = rows;
  g->cols = cols;
  g->nnz = nnz;
  int r = 0;
  g->row_off[0] = 0;
  for (int i = 0; i < nnz; ++i) {
    while (e[i].row != r) g->row_off[++r] = (uint16_t)i;
    g->col[i] = e[i].col;
    for (int s = 0; s < 8; ++s) g->vij[s][i] = e[i].v[s];
  }
  while (r < rows) g->row_off[++r] = (uint16_t)nnz;
  for (int k = 0; k < rows; ++k) g->degree[k] = (uint8_t)(g->row_off[k + 1] - g->row_off[k]);
}

void init_graphs() {
  build_graph(&g_bg[0], 1, kBG1Edges, NRLDPC_BG1_NNZ, NRLDPC_BG1_ROWS, NRLDPC_BG1_COLS);
  build_graph(&g_bg[1], 2, kBG2Edges, NRLDPC_BG2_NNZ, NRLDPC_BG2_ROWS, NRLDPC_BG2_COLS);
}

struct CrcSpec {
  int width;
  uint32_t poly;
};

bool crc_spec(int crctype, CrcSpec* s) {
  switch (crctype) {
    case 0: *s = {16, 0x1021u}; return true;      // CRC16
    case 1: *s = {24, 0x864CFBu}; return true;    // CRC24A
    case 2: *s = {24, 0x800063u}; return true;    // CRC24B
    case 3: *s = {24, 0xB2B117u}; return true;    // CRC24C
    default: return false;
  }
}

// Multiply a remainder by x modulo g(x).
inline uint32_t mulx(uint32_t r, const CrcSpec& s) {
  const uint32_t top = 1u << (s.width - 1);
  const uint32_t mask = (s.width == 32) ? 0xFFFFFFFFu : ((1u << s.width) - 1u);
  return ((r & top) ? ((r << 1) ^ s.poly) : (r << 1)) & mask;
}

}  // namespace

const BaseGraph& base_graph(int bgn) {
  std::call_once(g_bg_once, init_graphs);
  return g_bg[bgn == 1 ? 0 : 1];
}

// Kb rule of TS 38.212 5.2.2 and smallest Zc with Kb*Zc >= B
// (c_lib/ldpc_internal.c:24-64).
static void pick_lifting(int B, int bgn, int* Zc, int* iLS) {
  int Kb;
  if (bgn == 1) {
    Kb = 22;
  } else if (B > 640) {
    Kb = 10;
  } else if (B > 560) {
    Kb = 9;
  } else if (B > 192) {
    Kb = 8;
  } else {
    Kb = 6;
  }
  int best = 0xFFFF, set = -1;
  for (int s = 0; s < 8; ++s) {
    for (int j = 0; j < 8 && kLiftingSets[s][j]; ++j) {
      const int z = kLiftingSets[s][j];
      if (Kb * z >= B) {
        if (z < best) {
          best = z;
          set = s;
        }
        break;
      }
    }
  }
  *Zc = best;
  *iLS = set;
}

int derive_params(const ldpc_in_config_t& in, CodeParams* p, bool verbose) {
  memset(p, 0, sizeof(*p));
  p->bgn = in.bgn;
  p->A = in.A;
  p->crctype = in.crctype;
  p->E = in.E;
  p->rv = in.rv;
  p->Qm = in.Qm;
  p->harq_on = in.HARQ_on;
  const char* why = nullptr;
  if (in.bgn != 1 && in.bgn != 2) {
    why = "base graph number must be 1 or 2";
  } else if (in.crctype > 3) {
    why = "CRC type must be 0..3";
  } else if (in.Qm != 1 && in.Qm != 2 && in.Qm != 4 && in.Qm != 6 && in.Qm != 8) {
    why = "modulation order must be 1, 2, 4, 6 or 8";
  } else if (in.HARQ_on > 1) {
    why = "HARQ_on must be 0 or 1";
  } else if (in.rv > 3) {
    why = "redundancy version must be 0..3";
  } else if (in.E % in.Qm != 0) {
    why = "E must be a multiple of Qm";
  } else if (in.A % 8 != 0) {
    why = "A must be a multiple of 8";
  }
  if (!why) {
    // B is kept in 16 bits exactly as the reference's uint16_t field.
    p->B = (uint16_t)(in.A + (in.crctype == 0 ? 16 : 24));
    if (in.bgn == 1 && p->B > 8448) why = "BG1 needs B <= 8448";
    if (in.bgn == 2 && p->B > 3840) why = "BG2 needs B <= 3840";
  }
  if (why) {
    if (verbose) {
      fprintf(stderr, "nrldpc: invalid LDPC configuration (%s): bgn=%d A=%d crctype=%d E=%d rv=%d Qm=%d HARQ_on=%d\n",
              why, in.bgn, in.A, in.crctype, in.E, in.rv, in.Qm, in.HARQ_on);
    }
    return -1;
  }
  pick_lifting(p->B, p->bgn, &p->Zc, &p->iLS);
  const BaseGraph& g = base_graph(p->bgn);
  p->rows = g.rows;
  p->cols = g.cols;
  p->nnz = g.nnz;
  if (p->bgn == 1) {
    p->K = 22 * p->Zc;
    p->N = 66 * p->Zc;
  } else {
    p->K = 10 * p->Zc;
    p->N = 50 * p->Zc;
  }
  p->F = p->K - p->B;
  // TS 38.212 Table 5.4.2.1-2 with Ncb = N (c_lib/ldpc_internal.c:147-156).
  static const int k0_bg1[4] = {0, 17, 33, 56};
  static const int k0_bg2[4] = {0, 13, 25, 43};
  p->k0 = (p->bgn == 1 ? k0_bg1 : k0_bg2)[p->rv] * p->Zc;
  p->lq_len = p->N + 2 * p->Zc;
  p->Nv = p->N - p->F;
  const int fill_lo = p->B - 2 * p->Zc, fill_hi = p->K - 2 * p->Zc;
  p->c0 = p->k0 < fill_lo ? p->k0 : (p->k0 < fill_hi ? fill_lo : p->k0 - p->F);
  p->symbols = p->E / p->Qm;
  p->crc_w = p->crctype == 0 ? 16 : 24;
  return 0;
}

uint32_t crc_remainder(const uint8_t* data, int len, int crctype) {
  CrcSpec s;
  if (!crc_spec(crctype, &s)) return 0;
  // Byte table: entry v = v(x) * x^W mod g(x); MSB-first byte update.
  static uint32_t tab[4][256];
  static std::once_flag once;
  std::call_once(once, [] {
    for (int t = 0; t < 4; ++t) {
      CrcSpec st;
      crc_spec(t, &st);
      for (uint32_t v = 0; v < 256; ++v) {
        uint32_t r = v << (st.width - 8);
        for (int b = 0; b < 8; ++b) r = mulx(r, st);
        tab[t][v] = r;
      }
    }
  });
  const uint32_t mask = (1u << s.width) - 1u;
  uint32_t crc = 0;
  for (int i = 0; i < len; ++i) {
    const uint32_t idx = ((crc >> (s.width - 8)) ^ data[i]) & 0xFFu;
    crc = ((crc << 8) ^ tab[crctype][idx]) & mask;
  }
  return crc & mask;
}

void crc_position_table(int crctype, uint32_t* out) {
  CrcSpec s;
  if (!crc_spec(crctype, &s)) {
    memset(out, 0, sizeof(uint32_t) * kMaxB);
    return;
  }
  uint32_t r = 1;
  for (int i = 0; i < s.width; ++i) r = mulx(r, s);  // x^W mod g
  for (int d = 0; d < kMaxB; ++d) {
    out[d] = r;
    r = mulx(r, s);
  }
}

}  // namespace nrldpc
