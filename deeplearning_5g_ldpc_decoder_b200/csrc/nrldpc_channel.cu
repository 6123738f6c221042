// nrldpc_channel.cu — device LLR front-end: NR QAM mapping, complex AWGN,
// max-log demapping and int16 quantisation, for batches of code blocks.
//
// Restates the reference's test channel (c_lib/tx_rx_process.c:20-324):
//  * TS 38.211 5.1 constellations with the reference's float expressions
//    (bit_sign(b) = 1 - 2b, nested amplitude, times A = 1/sqrt(2|10|42|170)),
//  * piecewise-linear max-log LLRs per bit pair (:101-268), evaluated as
//    ((c1*A) * (s*r + c2*A)) / noise_var with the reference's segment
//    boundaries and strict "<" comparisons, round-to-nearest float ops,
//  * quantisation round(128*llr) (away from zero), clipped to +-10000 (:27-40).
// The noise comes from a counter-based generator (splitmix64 of seed, block,
// symbol; Box-Muller) instead of libc rand(); the noisy symbols can be returned
// so the demapper can be checked against a host restatement.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

// One segment of a piecewise max-log LLR: for r < thr*A (last: always),
// llr = (c1*A) * (s*r + c2*A) / noise_var.
struct Seg {
  float thr, c1, s, c2;
};
constexpr float kInf = 3.0e38f;

// Segment tables per bit pair (re/im share them), restating
// c_lib/tx_rx_process.c:101-231.
__constant__ Seg kQam16[2][3] = {
    {{-2, 8, 1, 1}, {2, 4, 1, 0}, {kInf, 8, 1, -1}},
    {{0, 4, 1, 2}, {kInf, 4, -1, 2}, {kInf, 0, 0, 0}},
};
__constant__ int kQam16N[2] = {3, 2};
__constant__ Seg kQam64[3][7] = {
    {{-6, 16, 1, 3}, {-4, 12, 1, 2}, {-2, 8, 1, 1}, {2, 4, 1, 0}, {4, 8, 1, -1}, {6, 12, 1, -2}, {kInf, 16, 1, -3}},
    {{-6, 8, 1, 5}, {-2, 4, 1, 4}, {0, 8, 1, 3}, {2, 8, -1, 3}, {6, 4, -1, 4}, {kInf, 8, -1, 5}, {kInf, 0, 0, 0}},
    {{-4, 4, 1, 6}, {0, 4, -1, -2}, {4, 4, 1, -2}, {kInf, 4, -1, 6}, {kInf, 0, 0, 0}, {kInf, 0, 0, 0},
     {kInf, 0, 0, 0}},
};
__constant__ int kQam64N[3] = {7, 6, 4};
__constant__ Seg kQam256[4][15] = {
    {{-14, 32, 1, 7}, {-12, 28, 1, 6}, {-10, 24, 1, 5}, {-8, 20, 1, 4}, {-6, 16, 1, 3}, {-4, 12, 1, 2},
     {-2, 8, 1, 1}, {2, 4, 1, 0}, {4, 8, 1, -1}, {6, 12, 1, -2}, {8, 16, 1, -3}, {10, 20, 1, -4},
     {12, 24, 1, -5}, {14, 28, 1, -6}, {kInf, 32, 1, -7}},
    {{-14, 16, 1, 11}, {-12, 12, 1, 10}, {-10, 8, 1, 9}, {-6, 4, 1, 8}, {-4, 8, 1, 7}, {-2, 12, 1, 6},
     {0, 16, 1, 5}, {2, 16, -1, 5}, {4, 12, -1, 6}, {6, 8, -1, 7}, {10, 4, -1, 8}, {12, 8, -1, 9},
     {14, 12, -1, 10}, {kInf, 16, -1, 11}, {kInf, 0, 0, 0}},
    {{-14, 8, 1, 13}, {-10, 4, 1, 12}, {-8, 8, 1, 11}, {-6, 8, -1, -5}, {-2, 4, -1, -4}, {0, 8, -1, -3},
     {2, 8, 1, -3}, {6, 4, 1, -4}, {8, 8, 1, -5}, {10, 8, -1, 11}, {14, 4, -1, 12}, {kInf, 8, -1, 13},
     {kInf, 0, 0, 0}, {kInf, 0, 0, 0}, {kInf, 0, 0, 0}},
    {{-12, 4, 1, 14}, {-8, 4, -1, -10}, {-4, 4, 1, 6}, {0, 4, -1, -2}, {4, 4, 1, -2}, {8, 4, -1, 6},
     {12, 4, 1, -10}, {kInf, 4, -1, 14}, {kInf, 0, 0, 0}, {kInf, 0, 0, 0}, {kInf, 0, 0, 0}, {kInf, 0, 0, 0},
     {kInf, 0, 0, 0}, {kInf, 0, 0, 0}, {kInf, 0, 0, 0}},
};
__constant__ int kQam256N[4] = {15, 14, 12, 8};

__device__ __forceinline__ float seg_llr(const Seg* seg, int n, float r, float A, float nv) {
  int k = 0;
  while (k < n - 1 && !(r < __fmul_rn(seg[k].thr, A))) ++k;
  const Seg s = seg[k];
  const float lin = __fadd_rn(__fmul_rn(s.s, r), __fmul_rn(s.c2, A));
  return __fdiv_rn(__fmul_rn(__fmul_rn(s.c1, A), lin), nv);
}

__device__ __forceinline__ int16_t quantize(float llr) {
  const float scaled = __fmul_rn(llr, 128.0f);
  int32_t q = (int32_t)(scaled >= 0.0f ? __fadd_rn(scaled, 0.5f) : __fsub_rn(scaled, 0.5f));
  q = q > 10000 ? 10000 : (q < -10000 ? -10000 : q);
  return (int16_t)q;
}

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float bsign(uint32_t b) { return b ? -1.0f : 1.0f; }

__global__ void channel_kernel(const uint8_t* __restrict__ rm, int64_t rm_stride, int32_t num_cw, int32_t E,
                               int32_t Qm, float nv, float sigma, float A, uint64_t seed,
                               int16_t* __restrict__ llr, int64_t llr_stride, float* __restrict__ symbols) {
  const int64_t nsym = E / Qm;
  const int64_t total = nsym * (int64_t)num_cw;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cw = g / nsym, s = g - cw * nsym;
    const uint8_t* in = rm + cw * rm_stride;
    uint32_t b[8];
    for (int j = 0; j < Qm; ++j) {
      const int64_t t = s * Qm + j;
      b[j] = (in[t >> 3] >> (7 - (t & 7))) & 1u;
    }
    float re, im;
    if (Qm == 1) {
      re = im = __fmul_rn(bsign(b[0]), A);
    } else if (Qm == 2) {
      re = __fmul_rn(bsign(b[0]), A);
      im = __fmul_rn(bsign(b[1]), A);
    } else if (Qm == 4) {
      re = __fmul_rn(__fmul_rn(bsign(b[0]), __fsub_rn(2.0f, bsign(b[2]))), A);
      im = __fmul_rn(__fmul_rn(bsign(b[1]), __fsub_rn(2.0f, bsign(b[3]))), A);
    } else if (Qm == 6) {
      re = __fmul_rn(__fmul_rn(bsign(b[0]), __fsub_rn(4.0f, __fmul_rn(bsign(b[2]), __fsub_rn(2.0f, bsign(b[4]))))), A);
      im = __fmul_rn(__fmul_rn(bsign(b[1]), __fsub_rn(4.0f, __fmul_rn(bsign(b[3]), __fsub_rn(2.0f, bsign(b[5]))))), A);
    } else {
      re = __fmul_rn(__fmul_rn(bsign(b[0]), __fsub_rn(8.0f, __fmul_rn(bsign(b[2]), __fsub_rn(4.0f,
                     __fmul_rn(bsign(b[4]), __fsub_rn(2.0f, bsign(b[6]))))))), A);
      im = __fmul_rn(__fmul_rn(bsign(b[1]), __fsub_rn(8.0f, __fmul_rn(bsign(b[3]), __fsub_rn(4.0f,
                     __fmul_rn(bsign(b[5]), __fsub_rn(2.0f, bsign(b[7]))))))), A);
    }
    // Box-Muller from a counter-based generator.
    const uint64_t z = splitmix(seed ^ splitmix(((uint64_t)cw << 32) ^ (uint64_t)s));
    const float u1 = ((float)(z >> 40) + 1.0f) * (1.0f / 16777218.0f);
    const float u2 = ((float)((z >> 16) & 0xFFFFFFu) + 1.0f) * (1.0f / 16777218.0f);
    const float rad = sqrtf(-2.0f * logf(u1));
    float sn, cs;
    sincospif(2.0f * u2, &sn, &cs);
    re = __fadd_rn(re, __fmul_rn(sigma, __fmul_rn(rad, cs)));
    im = __fadd_rn(im, __fmul_rn(sigma, __fmul_rn(rad, sn)));
    if (symbols) {
      symbols[2 * g] = re;
      symbols[2 * g + 1] = im;
    }
    int16_t* out = llr + cw * llr_stride + s * Qm;
    if (Qm == 1) {
      out[0] = quantize(__fdiv_rn(__fmul_rn(__fmul_rn(4.0f, __fadd_rn(re, im)), A), nv));
    } else if (Qm == 2) {
      out[0] = quantize(__fdiv_rn(__fmul_rn(__fmul_rn(4.0f, re), A), nv));
      out[1] = quantize(__fdiv_rn(__fmul_rn(__fmul_rn(4.0f, im), A), nv));
    } else if (Qm == 4) {
      for (int p = 0; p < 2; ++p) {
        out[2 * p] = quantize(seg_llr(kQam16[p], kQam16N[p], re, A, nv));
        out[2 * p + 1] = quantize(seg_llr(kQam16[p], kQam16N[p], im, A, nv));
      }
    } else if (Qm == 6) {
      for (int p = 0; p < 3; ++p) {
        out[2 * p] = quantize(seg_llr(kQam64[p], kQam64N[p], re, A, nv));
        out[2 * p + 1] = quantize(seg_llr(kQam64[p], kQam64N[p], im, A, nv));
      }
    } else {
      for (int p = 0; p < 4; ++p) {
        out[2 * p] = quantize(seg_llr(kQam256[p], kQam256N[p], re, A, nv));
        out[2 * p + 1] = quantize(seg_llr(kQam256[p], kQam256N[p], im, A, nv));
      }
    }
  }
}

}  // namespace

int launch_channel(const uint8_t* rm, int64_t rm_stride, int32_t num_cw, int32_t E, int32_t Qm, float nv,
                   float sigma, float A, uint64_t seed, int16_t* llr, int64_t llr_stride, float* symbols,
                   void* stream) {
  const int64_t total = (int64_t)(E / Qm) * num_cw;
  if (total == 0) return 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (total + 255) / 256;
  const int grid = (int)(want < 16LL * sms ? want : 16LL * sms);
  channel_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(rm, rm_stride, num_cw, E, Qm, nv, sigma,
                                                                           A, seed, llr, llr_stride, symbols);
  count_launch();
  return (int)cudaGetLastError();
}

}  // namespace nrldpc
