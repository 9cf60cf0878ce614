// Wire encoding of dedispersed rows (sm_100a): the per-tile quantiser of
// TransportTx._encode_rows (src/dsart/transport/tx.py:825-873).
//
// A row is one tile of one DM row: n_filled complex cells.
//   cint8 (16 bits per cell): amax = max |re|, |im| over the row (float32,
//     exact); scale = float32(double(amax) / 127), 1 for an all-zero row;
//     inv = float32(1 / double(scale)); q = clip(rint(x * inv), -128, 127)
//     with x * inv a float32 product and rint ties-to-even.
//   cfp16 (32 bits per cell): each part rounded to nearest-even half;
//     scale 1.
// One CTA per row: a max reduction, then the quantise pass over the row.
#include "dsb_common.cuh"

#include <algorithm>

namespace {

constexpr int ENC_THREADS = 256;

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

__global__ void __launch_bounds__(ENC_THREADS) encode_cint8_kernel(
    const float2* __restrict__ rows, long long row_stride, int n_filled,
    char2* __restrict__ q, float* __restrict__ scales) {
  __shared__ float s_max[ENC_THREADS / 32];
  __shared__ float s_inv;
  const long long r = blockIdx.x;
  const float2* row = rows + r * row_stride;
  float m = 0.f;
  for (int i = threadIdx.x; i < n_filled; i += ENC_THREADS) {
    const float2 v = row[i];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.f;
    for (int w = 0; w < ENC_THREADS / 32; ++w) a = fmaxf(a, s_max[w]);
    const float scale = a == 0.f ? 1.f : (float)((double)a / 127.0);
    scales[r] = scale;
    s_inv = (float)(1.0 / (double)scale);
  }
  __syncthreads();
  const float inv = s_inv;
  char2* out = q + r * (long long)n_filled;
  for (int i = threadIdx.x; i < n_filled; i += ENC_THREADS) {
    const float2 v = row[i];
    const float a = fminf(fmaxf(rintf(v.x * inv), -128.f), 127.f);
    const float b = fminf(fmaxf(rintf(v.y * inv), -128.f), 127.f);
    out[i] = make_char2((signed char)(int)a, (signed char)(int)b);
  }
}

__global__ void encode_cfp16_kernel(const float2* __restrict__ rows, long long row_stride,
                                    int n_rows, int n_filled, __half2* __restrict__ q,
                                    float* __restrict__ scales) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (long long r = first; r < n_rows; r += stride) scales[r] = 1.f;
  const long long n = (long long)n_rows * n_filled;
  for (long long e = first; e < n; e += stride) {
    const long long r = e / n_filled, i = e - r * n_filled;
    const float2 v = rows[r * row_stride + i];
    q[e] = __floats2half2_rn(v.x, v.y);
  }
}

}  // namespace

extern "C" {

int dsb_encode_rows(const void* rows, long long row_stride, int n_rows, int n_filled,
                    int bits_per_cell, void* payload, float* scales, cudaStream_t stream) {
  if (((!rows || !payload) && n_filled > 0) || !scales || n_rows < 0 || n_filled < 0 ||
      row_stride < n_filled)
    return DSB_E_ARG;
  if (bits_per_cell != 16 && bits_per_cell != 32) return DSB_E_UNSUPPORTED;
  if (n_rows == 0) return DSB_OK;
  if (bits_per_cell == 16) {
    encode_cint8_kernel<<<n_rows, ENC_THREADS, 0, stream>>>(
        (const float2*)rows, row_stride, n_filled, (char2*)payload, scales);
  } else {
    const long long n = std::max<long long>((long long)n_rows * n_filled, n_rows);
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    encode_cfp16_kernel<<<blocks, 256, 0, stream>>>((const float2*)rows, row_stride, n_rows,
                                                    n_filled, (__half2*)payload, scales);
  }
  return launch_status();
}

}  // extern "C"
