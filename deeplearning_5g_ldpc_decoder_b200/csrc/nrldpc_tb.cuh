// nrldpc_tb.cuh — transport-block arithmetic shared by host and device:
// code-block segmentation (TS 38.212 5.2.2), the per-code-block rate-matching
// lengths (5.4.2.1), lifting-size selection, and the derived parameters of one
// code block in the form the decode kernels use.
//
// The per-code-block configuration is expressed as the reference's
// ldpc_in_config_t (bgn, A, crctype, E, rv, Qm): A is the code block's
// information bits before its CRC and crctype its CRC (CRC24B when the
// transport block has several code blocks, else the transport-block CRC), so
// every code block decodes exactly like a single-block call of the reference
// (c_lib/ldpc_internal.c:66-170 derives the same B, Zc, K, F, N, k0).
#pragma once

#include <stdint.h>

namespace nrldpc {

struct TbSeg {
  int32_t bgn;      // base graph
  int32_t L_tb;     // transport-block CRC length (16 or 24)
  int32_t B;        // A + L_tb
  int32_t C;        // code blocks
  int32_t Kp;       // K': bits per code block before filler (information + CB CRC)
  int32_t Zc, iLS;  // lifting size and its set index
  int32_t A_cb;     // code-block information bits (the reference's A field)
  int32_t crc_cb;   // code-block CRC type: 0 CRC16, 1 CRC24A, 2 CRC24B
  int32_t E_lo, E_hi, n_lo;   // code blocks 0..n_lo-1 carry E_lo bits, the rest E_hi
  int32_t N;        // mother code length after puncturing (66 Zc / 50 Zc)
  int32_t Ncb;      // circular-buffer length: N, or N_ref with limited-buffer rate matching
};

// Error codes of tb_segment (0 = valid).
enum TbSegError : int32_t {
  kTbOk = 0,
  kTbBadArg = 1,         // A not a positive multiple of 8, bad Qm / rv / bgn, G not a multiple of Qm
  kTbNotDivisible = 2,   // B + C*L not divisible into equal byte-aligned code blocks (TS 38.214 TBS rule)
  kTbTooLong = 3,        // a code block's E does not fit the 16-bit E field
  kTbTooShort = 4,       // a code block would get no coded bits
  kTbLbrm = 5,           // the limited circular buffer would cut into the systematic bits
};

// Smallest lifting size Z = a * 2^j <= 384 (a = 2,3,5,7,9,11,13,15; set index
// iLS = position of a) with Kb * Z >= K (TS 38.212 Table 5.3.2-1).
__host__ __device__ inline void tb_lifting(int K, int Kb, int* Zc, int* iLS) {
  const int base[8] = {2, 3, 5, 7, 9, 11, 13, 15};
  int best = 1 << 30, set = -1;
  for (int s = 0; s < 8; ++s) {
    int z = base[s];
    while (Kb * z < K && z * 2 <= 384) z *= 2;
    if (Kb * z >= K && z < best) {
      best = z;
      set = s;
    }
  }
  *Zc = best;
  *iLS = set;
}

// Code-block segmentation of a transport block of A payload bits coded into G
// bits with modulation order Qm on base graph bgn (one layer).  tbs_lbrm > 0
// turns on limited-buffer rate matching (TS 38.212 5.4.2.1): every code block's
// circular buffer is Ncb = min(N, N_ref), N_ref = floor(TBS_LBRM / (C R_LBRM)),
// R_LBRM = 2/3.
__host__ __device__ inline int32_t tb_segment(int32_t A, int32_t G, int32_t Qm, int32_t bgn, int32_t tbs_lbrm,
                                              TbSeg* s) {
  if (A <= 0 || (A & 7) || (bgn != 1 && bgn != 2) || !(Qm == 1 || Qm == 2 || Qm == 4 || Qm == 6 || Qm == 8) ||
      G <= 0 || G % Qm)
    return kTbBadArg;
  s->bgn = bgn;
  s->L_tb = A > 3824 ? 24 : 16;
  s->B = A + s->L_tb;
  const int Kcb = bgn == 1 ? 8448 : 3840;
  int Bp;
  if (s->B <= Kcb) {
    s->C = 1;
    Bp = s->B;
  } else {
    s->C = (s->B + (Kcb - 24) - 1) / (Kcb - 24);
    Bp = s->B + 24 * s->C;
  }
  if (Bp % s->C) return kTbNotDivisible;
  s->Kp = Bp / s->C;
  int Kb = 22;
  if (bgn == 2) Kb = s->B > 640 ? 10 : (s->B > 560 ? 9 : (s->B > 192 ? 8 : 6));
  tb_lifting(s->Kp, Kb, &s->Zc, &s->iLS);
  if (s->C == 1) {
    s->A_cb = A;
    s->crc_cb = s->L_tb == 16 ? 0 : 1;
  } else {
    s->A_cb = s->Kp - 24;
    s->crc_cb = 2;
    if (s->A_cb & 7) return kTbNotDivisible;
  }
  s->N = (bgn == 1 ? 66 : 50) * s->Zc;
  s->Ncb = s->N;
  if (tbs_lbrm > 0) {
    const int64_t nref = (3 * (int64_t)tbs_lbrm) / (2 * (int64_t)s->C);
    if (nref < s->N) s->Ncb = (int32_t)nref;
    if (s->Ncb < ((bgn == 1 ? 22 : 10) - 2) * s->Zc) return kTbLbrm;
  }
  const int q = G / Qm;   // symbols (one layer)
  s->E_lo = Qm * (q / s->C);
  s->E_hi = Qm * ((q + s->C - 1) / s->C);
  s->n_lo = s->C - q % s->C;
  if (s->E_lo <= 0) return kTbTooShort;
  if (s->E_hi > 65535) return kTbTooLong;
  return kTbOk;
}

// Rate-matched length and first LLR of code block r.
__host__ __device__ inline int32_t tb_cb_E(const TbSeg& s, int r) { return r < s.n_lo ? s.E_lo : s.E_hi; }
__host__ __device__ inline int64_t tb_cb_llr_start(const TbSeg& s, int r) {
  return r < s.n_lo ? (int64_t)r * s.E_lo : (int64_t)s.n_lo * s.E_lo + (int64_t)(r - s.n_lo) * s.E_hi;
}

// Derived rate-recovery parameters of one code block (the fields of
// gen_ldpc_parameters the decode kernels use).  With Ncb = N they are the
// reference's; with a limited buffer k0 = floor(f_rv Ncb / (N_bg Zc)) Zc
// (TS 38.212 Table 5.4.2.1-2) and only Ncb - F positions take coded bits.
struct CbDerived {
  int32_t B, K, N, F, Nv, c0, k0, symbols, Ncb;
};
__host__ __device__ inline CbDerived tb_cb_derive(const TbSeg& s, int32_t E, int32_t rv, int32_t Qm) {
  CbDerived d;
  d.B = s.Kp;
  d.K = (s.bgn == 1 ? 22 : 10) * s.Zc;
  d.N = (s.bgn == 1 ? 66 : 50) * s.Zc;
  d.F = d.K - d.B;
  const int k0_bg1[4] = {0, 17, 33, 56};
  const int k0_bg2[4] = {0, 13, 25, 43};
  const int f = s.bgn == 1 ? k0_bg1[rv & 3] : k0_bg2[rv & 3];
  d.Ncb = s.Ncb;
  d.k0 = (int32_t)(((int64_t)f * s.Ncb) / ((int64_t)(s.bgn == 1 ? 66 : 50) * s.Zc)) * s.Zc;
  d.Nv = d.Ncb - d.F;
  const int fill_lo = d.B - 2 * s.Zc, fill_hi = d.K - 2 * s.Zc;
  d.c0 = d.k0 < fill_lo ? d.k0 : (d.k0 < fill_hi ? fill_lo : d.k0 - d.F);
  d.symbols = E / Qm;
  return d;
}

// Graph key of a (BG, Zc): (bgn-1)*64 + iLS*8 + log2(Zc / base(iLS)); 128 keys.
__host__ __device__ inline int tb_graph_key(int bgn, int Zc, int iLS) {
  const int base[8] = {2, 3, 5, 7, 9, 11, 13, 15};
  int j = 0;
  while ((base[iLS] << j) < Zc) ++j;
  return (bgn - 1) * 64 + iLS * 8 + j;
}

}  // namespace nrldpc
