// nrldpc_encode.cu — batched 5G NR LDPC encoder + rate matching for sm_100a.
//
// Restates the reference's transmit chain (c_lib/c_ldpc_5g_encoder.c:66-88):
//  * CRC attach (calculate_crc over A/8 payload bytes, MSB first),
//  * QC-LDPC encoding (c_lib/ldpc_encoder.c:52-242): syndromes of the first
//    four base-graph rows over the systematic part, the double-diagonal core
//    parity solve (pc0 from the summed syndromes through the I2 / I4
//    circulant, pc1/pc3 through I1 / I3, pc2 from row 2 / row 1), then every
//    extension row's parity as a plain XOR over systematic + core columns,
//  * bit selection from k0 over the circular buffer without filler bits and
//    the Qm row/column interleave, packed MSB first
//    (c_lib/ldpc_rate_match.c:27-106).
// One CTA per code block; the codeword is staged as one byte per bit in shared
// memory (at most 68*384 bytes).  It exists to serve the reference's encode
// symbol and to produce test vectors on the device; it is not on the decode
// hot path.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_internal.h"

namespace nrldpc {

namespace {

constexpr int kEncThreads = 384;

__global__ void __launch_bounds__(kEncThreads) encode_kernel(const __grid_constant__ EncodeParams p) {
  extern __shared__ uint8_t s_cw[];              // [cols*Zc] codeword bits, one per byte
  __shared__ uint8_t s_L[4][kMaxZc];
  __shared__ uint32_t s_crc;
  const int tid = threadIdx.x;
  const int Zc = p.Zc;
  for (int cw = blockIdx.x; cw < p.num_cw; cw += gridDim.x) {
    const uint8_t* info = p.info + (int64_t)cw * p.info_stride;
    if (tid == 0) s_crc = 0u;
    __syncthreads();
    // Payload bits and the CRC remainder sum_i bit_i * x^(A-1-i+W) mod g(x).
    for (int base = 0; base < p.A; base += blockDim.x) {
      const int i = base + tid;
      uint32_t t = 0u;
      if (i < p.A) {
        const uint8_t bit = (info[i >> 3] >> (7 - (i & 7))) & 1u;
        s_cw[i] = bit;
        if (bit) t = __ldg(p.crc_tab + (p.A - 1 - i));
      }
      t = __reduce_xor_sync(0xFFFFFFFFu, t);
      if ((tid & 31) == 0 && t) atomicXor(&s_crc, t);
    }
    __syncthreads();
    const int L = p.B - p.A;
    for (int i = tid; i < p.K - p.A; i += blockDim.x)
      s_cw[p.A + i] = i < L ? (uint8_t)((s_crc >> (L - 1 - i)) & 1u) : (uint8_t)0;   // CRC then filler zeros
    __syncthreads();
    // Syndromes of rows 0..3 over the information + filler columns.
    for (int k = tid; k < 4 * Zc; k += blockDim.x) {
      const int r = k / Zc, zx = k - r * Zc;
      uint8_t s = 0;
      for (int e = p.row_off[r]; e < p.row_off[r + 1]; ++e) {
        const uint32_t ed = p.edge[e];
        const int col = (int)(ed & 0xFFFFu), sh = (int)(ed >> 16);
        if (col < p.Kb) {
          int idx = sh + zx;
          idx = idx >= Zc ? idx - Zc : idx;
          s ^= s_cw[col * Zc + idx];
        }
      }
      s_L[r][zx] = s;
    }
    __syncthreads();
    uint8_t* w = s_cw + p.K;      // parity groups follow the K systematic bits
    for (int zx = tid; zx < Zc; zx += blockDim.x) {
      int idx = p.shift1 + zx;
      idx = idx >= Zc ? idx - Zc : idx;
      w[idx] = s_L[0][zx] ^ s_L[1][zx] ^ s_L[2][zx] ^ s_L[3][zx];          // pc0 = I2^-1 / I4^-1 applied
    }
    __syncthreads();
    for (int zx = tid; zx < Zc; zx += blockDim.x) {
      int idx = p.shift0 + zx;
      idx = idx >= Zc ? idx - Zc : idx;
      const uint8_t t = w[idx];
      w[Zc + zx] = s_L[0][zx] ^ t;           // pc1
      w[3 * Zc + zx] = s_L[3][zx] ^ t;       // pc3
    }
    __syncthreads();
    for (int zx = tid; zx < Zc; zx += blockDim.x)
      w[2 * Zc + zx] = p.bgn == 1 ? (uint8_t)(s_L[2][zx] ^ w[3 * Zc + zx]) : (uint8_t)(s_L[1][zx] ^ w[Zc + zx]);
    __syncthreads();
    // Extension rows: each parity bit is the XOR over systematic + core columns.
    for (int k = tid; k < (p.R - 4) * Zc; k += blockDim.x) {
      const int r = 4 + k / Zc, zx = k % Zc;
      uint8_t s = 0;
      for (int e = p.row_off[r]; e < p.row_off[r + 1]; ++e) {
        const uint32_t ed = p.edge[e];
        const int col = (int)(ed & 0xFFFFu), sh = (int)(ed >> 16);
        if (col < p.Kb + 4) {
          int idx = sh + zx;
          idx = idx >= Zc ? idx - Zc : idx;
          s ^= s_cw[col * Zc + idx];
        }
      }
      w[r * Zc + zx] = s;
    }
    __syncthreads();
    // Rate matching: output bit t = s*Qm + b carries e[b*(E/Qm) + s], and
    // e[k] is circular-buffer position (c0 + k) mod (N-F) of the buffer
    // without filler bits, i.e. codeword bit 2Zc + position (+F past the filler).
    uint8_t* out = p.rm + (int64_t)cw * p.rm_stride;
    const int nbytes = (p.E + 7) >> 3;
    for (int y = tid; y < nbytes; y += blockDim.x) {
      uint32_t v = 0u;
      for (int b = 0; b < 8; ++b) {
        const int t = y * 8 + b;
        uint32_t bit = 0u;
        if (t < p.E) {
          const int sym = t / p.Qm, q = t - sym * p.Qm;
          const int k = q * p.symbols + sym;
          const int c = (p.c0 + k) % p.Nv;
          const int pos = c < p.B - 2 * Zc ? c : c + p.F;
          bit = s_cw[pos + 2 * Zc];
        }
        v |= bit << (7 - b);
      }
      out[y] = (uint8_t)v;
    }
    __syncthreads();
  }
}

}  // namespace

int launch_encode(const EncodeParams& p, void* stream) {
  const int smem = p.cols * p.Zc;
  cudaError_t e = cudaFuncSetAttribute(encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = p.num_cw < 8 * sms ? p.num_cw : 8 * sms;
  encode_kernel<<<grid, kEncThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(p);
  count_launch();
  return (int)cudaGetLastError();
}

}  // namespace nrldpc
