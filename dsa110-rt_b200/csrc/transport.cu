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
//
// dsb_ring_encode_cint8 applies the same cint8 quantiser to the stage-1
// output of one chunk and writes the int8 pairs straight into the stage-2
// ring at t + shift2, with each row's scale in a matching scale ring: the
// ring then holds what the search side of the reference receives.
#include "dsb_common.cuh"

#include <algorithm>

namespace {

constexpr int ENC_THREADS = 256;

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

// CTA-wide max of m; s_red holds one float per warp.  Every thread gets it.
template <int NT>
DSB_DEV float cta_max(float m, float* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = m;
  __syncthreads();
  float a = s_red[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) a = fmaxf(a, s_red[w]);
  return a;
}

// amax / 127 (1 for an all-zero row) in float32, through double as the
// reference's numpy code computes it
DSB_DEV float cint8_scale(float amax) {
  return amax == 0.f ? 1.f : (float)((double)amax / 127.0);
}
DSB_DEV float cint8_inv(float scale) { return (float)(1.0 / (double)scale); }

// one part: rint of the float32 product (ties to even), clipped to int8
DSB_DEV uint32_t cint8_part(float x, float inv) {
  return (uint32_t)(uint8_t)(int8_t)(int)fminf(fmaxf(rintf(x * inv), -128.f), 127.f);
}

__global__ void __launch_bounds__(ENC_THREADS) encode_cint8_kernel(
    const float2* __restrict__ rows, long long row_stride, int n_filled,
    char2* __restrict__ q, float* __restrict__ scales) {
  __shared__ float s_max[ENC_THREADS / 32];
  const long long r = blockIdx.x;
  const float2* row = rows + r * row_stride;
  float m = 0.f;
  for (int i = threadIdx.x; i < n_filled; i += ENC_THREADS) {
    const float2 v = row[i];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  const float scale = cint8_scale(cta_max<ENC_THREADS>(m, s_max));
  if (threadIdx.x == 0) scales[r] = scale;
  const float inv = cint8_inv(scale);
  uint16_t* out = reinterpret_cast<uint16_t*>(q) + r * (long long)n_filled;
  for (int i = threadIdx.x; i < n_filled; i += ENC_THREADS) {
    const float2 v = row[i];
    out[i] = (uint16_t)(cint8_part(v.x, inv) | cint8_part(v.y, inv) << 8);
  }
}

// Stage-1 rows of one chunk -> cint8 stage-2 ring.  One CTA per (time t,
// chgroup g x coarse DM d) row: X row at x_base[gd] + t * pitch[g] (complex64,
// n_filled[g] pattern cells, the rest of the pitch ignored); ring row at slot
// (t0 + t + shift2[gd]) mod seg_depth[gd] of segment seg_base[gd] (cells past
// n_filled written as 0); its scale at scales[sc_base[gd] + slot].
constexpr int RQ_THREADS = 128;

__global__ void __launch_bounds__(RQ_THREADS) ring_cint8_kernel(
    const float4* __restrict__ X, const long long* __restrict__ x_base,
    const int* __restrict__ pitch, const int* __restrict__ n_filled, int n_dm,
    const int* __restrict__ shift2, long long t0, uint32_t* __restrict__ D,
    const long long* __restrict__ seg_base, const int* __restrict__ seg_depth,
    float* __restrict__ scales, const long long* __restrict__ sc_base, int* status) {
  __shared__ float s_max[RQ_THREADS / 32];
  const int t = blockIdx.x, gd = blockIdx.y;
  const int g = gd / n_dm;
  const int pt = pitch[g], nf = n_filled[g];
  const long long xb = x_base[gd] + (long long)t * pt;
  const long long sb = seg_base[gd];
  const long long dep = seg_depth[gd];
  // two cells per 16-byte load and per 4-byte store
  if ((pt & 1) || (xb & 1) || (sb & 1) || nf < 0 || nf > pt || dep <= 0) {
    if (threadIdx.x == 0) dsb_flag(status, DSB_E_ARG);
    return;
  }
  long long slot = (t0 + t + shift2[gd]) % dep;
  if (slot < 0) slot += dep;
  const float4* row = X + xb / 2;
  const int np = pt / 2;
  float m = 0.f;
  for (int p = threadIdx.x; p < np; p += RQ_THREADS) {
    const float4 v = row[p];
    if (2 * p < nf) m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
    if (2 * p + 1 < nf) m = fmaxf(m, fmaxf(fabsf(v.z), fabsf(v.w)));
  }
  const float scale = cint8_scale(cta_max<RQ_THREADS>(m, s_max));
  if (threadIdx.x == 0) scales[sc_base[gd] + slot] = scale;
  const float inv = cint8_inv(scale);
  uint32_t* out = D + (sb + slot * pt) / 2;
  for (int p = threadIdx.x; p < np; p += RQ_THREADS) {
    const float4 v = row[p];
    uint32_t w = 0;
    if (2 * p < nf) w = cint8_part(v.x, inv) | cint8_part(v.y, inv) << 8;
    if (2 * p + 1 < nf) w |= cint8_part(v.z, inv) << 16 | cint8_part(v.w, inv) << 24;
    out[p] = w;
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

int dsb_ring_encode_cint8(const void* X, const long long* x_base, int n_t, const int* pitch,
                          const int* n_filled, int G, int n_dm, const int* shift2, long long t0,
                          void* D, const long long* seg_base, const int* seg_depth,
                          float* scales, const long long* sc_base, int* status,
                          cudaStream_t stream) {
  if (!X || !x_base || !pitch || !n_filled || !shift2 || !D || !seg_base || !seg_depth ||
      !scales || !sc_base || !status || n_t < 0 || G <= 0 || n_dm <= 0)
    return DSB_E_ARG;
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(D) & 3))
    return DSB_E_ARG;
  if ((long long)G * n_dm > 65535) return DSB_E_UNSUPPORTED;
  if (n_t == 0) return DSB_OK;
  ring_cint8_kernel<<<dim3(n_t, G * n_dm), RQ_THREADS, 0, stream>>>(
      (const float4*)X, x_base, pitch, n_filled, n_dm, shift2, t0, (uint32_t*)D, seg_base,
      seg_depth, scales, sc_base, status);
  return launch_status();
}

}  // extern "C"
