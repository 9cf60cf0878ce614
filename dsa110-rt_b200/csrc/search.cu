// Search side: fine-DM combine, image masking, boxcar detector, Layer-1
// noise estimate, and the FP64 uv-cell geometry kernel (sm_100a).
#include "dsb_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <type_traits>

#include <algorithm>

namespace {

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

// ===========================================================================
// uv cells (FP64): ix = rint(-(d / (c / (nu*1e9))) / cell) + N/2
// (grid/sparsity_pattern.py:1090-1170, same operation order as numpy)
// ===========================================================================
__global__ void uv_cells_kernel(const double* __restrict__ du, const double* __restrict__ dv,
                                int n_bl, const double* __restrict__ nu_ghz, int n_ch,
                                double cell_lambda, int half, int* __restrict__ row,
                                int* __restrict__ col) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_bl * n_ch) return;
  const int b = (int)(idx / n_ch), c = (int)(idx % n_ch);
  const double wl = 299792458.0 / (nu_ghz[c] * 1e9);
  const double u = -(du[b] / wl);
  const double v = -(dv[b] / wl);
  col[idx] = (int)rint(u / cell_lambda) + half;
  row[idx] = (int)rint(v / cell_lambda) + half;
}

// ===========================================================================
// Pipeline combine: Hermitian half-spectrum from stage-2 rings.
//   G_h[f, t, u, w] = 0.5 * sum_e sign_e(D[row_e(f)][t - sf[f, g_e]]) * (-1)^(u+w)
// where each entry e of half-cell (u, w) names a chgroup g, a cell inside
// that chgroup's pattern, and whether it is the conjugate mirror.
// ===========================================================================
struct CombArgs {
  const void* D;         // ring: complex64 (FMT 0), bf16 re/im pairs in 32 bits (1),
                         // or int8 re/im pairs in 16 bits (2) times the row's scale
  const float* scales;   // FMT 2: scales[sc_base[gc] + slot] of each ring row
  const long long* sc_base;
  const long long* seg_base;  // (G * n_coarse) ring segment of (chgroup, coarse DM)
  const int* seg_depth;       // (G * n_coarse) time slots of each segment
  int n_coarse;
  const int* hc_off;     // (n_half_cells + 1) CSR over half cells (u-major)
  const int* e_g;        // chgroup
  const int* e_cell;     // cell within the chgroup (negative = mirror, stored as ~cell)
  const int* d_pitch;    // (G) cells (row pitch) of each chgroup's segments
  const int* sfine;      // (n_fine_total, G) signed shifts
  const int* f2c;        // (n_fine_total) coarse index
  int f0, n_f, G, N;
  long long t0;          // stream time of output t = 0
  int n_t;
  int fftshift;
  float2* out;           // (n_f, n_t, N, N/2+1)
};

// One thread per (half cell, fine DM); time is walked in tiles of CB_T
// samples so every ring row is read sequentially (L1 sector reuse) and each
// output time is written coalesced across the half cells of a warp.
constexpr int CB_T = 8;

template <int FMT>
__global__ void __launch_bounds__(128) combine_rows_kernel(const CombArgs A) {
  const int nh = A.N / 2 + 1;
  const int n_hc = A.N * nh;
  const int hc = blockIdx.x * blockDim.x + threadIdx.x;
  if (hc >= n_hc) return;
  const int fl = blockIdx.y;
  const int f = A.f0 + fl;
  const int c = A.f2c[f];
  const int u = hc / nh, w = hc % nh;
  const bool flip = A.fftshift && ((u + w) & 1);
  float2* out = A.out + (size_t)fl * A.n_t * n_hc + hc;
  const int j0 = A.hc_off[hc], j1 = A.hc_off[hc + 1];
  for (int tt = 0; tt < A.n_t; tt += CB_T) {
    double re[CB_T], im[CB_T];
#pragma unroll
    for (int i = 0; i < CB_T; ++i) re[i] = im[i] = 0.0;
    for (int j = j0; j < j1; ++j) {
      const int g = A.e_g[j];
      int cell = A.e_cell[j];
      const bool mirror = cell < 0;
      if (mirror) cell = ~cell;
      const int gc = g * A.n_coarse + c;
      const long long ts0 = A.t0 + tt - A.sfine[(long long)f * A.G + g];
      const long long e0 = A.seg_base[gc] + cell;
      const long long dep = A.seg_depth[gc];
      const long long pitch = A.d_pitch[g];
      long long slot0 = ts0 % dep;
      if (slot0 < 0) slot0 += dep;
#pragma unroll
      for (int i = 0; i < CB_T; ++i) {
        long long slot = slot0 + i;
        if (slot >= dep) slot -= dep;
        float2 x;
        if constexpr (FMT == 2) {
          const char2 q = static_cast<const char2*>(A.D)[e0 + slot * pitch];
          const float sc = A.scales[A.sc_base[gc] + slot];
          x = make_float2(sc * (float)q.x, sc * (float)q.y);
        } else if constexpr (FMT == 1)
          x = bf16_pair_to_f2(static_cast<const uint32_t*>(A.D)[e0 + slot * pitch]);
        else
          x = static_cast<const float2*>(A.D)[e0 + slot * pitch];
        re[i] += x.x;
        im[i] += mirror ? -(double)x.y : (double)x.y;
      }
    }
#pragma unroll
    for (int i = 0; i < CB_T; ++i) {
      if (tt + i < A.n_t) {
        float o_re = (float)(0.5 * re[i]), o_im = (float)(0.5 * im[i]);
        if (flip) {
          o_re = -o_re;
          o_im = -o_im;
        }
        out[(size_t)(tt + i) * n_hc] = make_float2(o_re, o_im);
      }
    }
  }
}

// ===========================================================================
// Reference-layout dense cint8 combine (image/fused_combine_cuda.py:210-300,
// 560-700): streams [G, T_stream, 2, N, N] int8.  Calibrated forms add
// scale * q + offset per chgroup term, with one scale/offset per chgroup or
// (PER_T) per (chgroup, source time) [G, T_stream] -- the wire's per-tile
// scales (fused_combine_cuda.py:431-505).
// ===========================================================================
template <bool HALF, bool CALIB, bool OUT_F16, bool PER_T>
__global__ void combine_dense_kernel(const int8_t* __restrict__ streams,
                                     const int* __restrict__ shifts,
                                     const float* __restrict__ scales,
                                     const float* __restrict__ off_re,
                                     const float* __restrict__ off_im, void* __restrict__ out,
                                     int G, int t_stream, int t_det, int N, int t_lo,
                                     int fftshift) {
  const int nw = HALF ? N / 2 + 1 : N;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const int u = blockIdx.y * blockDim.y + threadIdx.y;
  const int t_out = blockIdx.z * blockDim.z + threadIdx.z;
  const int t = t_out + t_lo;
  if (w >= nw || u >= N || t >= t_det) return;
  const long long nsq = (long long)N * N;
  const int off_cell = u * N + w;
  const int off_m = ((N - u) % N) * N + ((N - w) % N);
  const long long t_stride = 2 * nsq, g_stride = (long long)t_stream * t_stride;
  float o_re, o_im;
  if (!CALIB) {
    int ar = 0, ai = 0, mr = 0, mi = 0;
    for (int g = 0; g < G; ++g) {
      const int ts = t - shifts[g];
      if (ts >= 0 && ts < t_stream) {
        const long long b = g * g_stride + ts * t_stride;
        ar += streams[b + off_cell];
        ai += streams[b + off_cell + nsq];
        if (HALF) {
          mr += streams[b + off_m];
          mi += streams[b + off_m + nsq];
        }
      }
    }
    if (HALF) {
      o_re = 0.5f * (float)(ar + mr);
      o_im = 0.5f * (float)(ai - mi);
    } else {
      o_re = (float)ar;
      o_im = (float)ai;
    }
  } else {
    float ar = 0.f, ai = 0.f, mr = 0.f, mi = 0.f;
    for (int g = 0; g < G; ++g) {
      const int ts = t - shifts[g];
      if (ts >= 0 && ts < t_stream) {
        const long long b = g * g_stride + ts * t_stride;
        const int gt = PER_T ? g * t_stream + ts : g;
        const float sc = scales[gt], orr = off_re[gt], oii = off_im[gt];
        ar = fmaf(sc, (float)streams[b + off_cell], ar) + orr;
        ai = fmaf(sc, (float)streams[b + off_cell + nsq], ai) + oii;
        if (HALF) {
          mr = fmaf(sc, (float)streams[b + off_m], mr) + orr;
          mi = fmaf(sc, (float)streams[b + off_m + nsq], mi) + oii;
        }
      }
    }
    if (HALF) {
      o_re = 0.5f * (ar + mr);
      o_im = 0.5f * (ai - mi);
    } else {
      o_re = ar;
      o_im = ai;
    }
  }
  if (fftshift && ((u + w) & 1)) {
    o_re = -o_re;
    o_im = -o_im;
  }
  const long long o = (long long)t_out * N * nw + (long long)u * nw + w;
  if (OUT_F16)
    reinterpret_cast<__half2*>(out)[o] = __floats2half2_rn(o_re, o_im);
  else
    reinterpret_cast<float2*>(out)[o] = make_float2(o_re, o_im);
}

// ===========================================================================
// image mask / normalise into the detector cube layout
//   cube[t, f, h, w] = img[f, t, h, w] * mask_f[f, h, w]
// ===========================================================================
template <bool OUT_F16>
__global__ void mask_to_cube_kernel(const float* __restrict__ img, const float* __restrict__ mask,
                                    int mask_per_f, int n_f, int n_t, int npix,
                                    void* __restrict__ cube, int cube_f_total, int cube_f0) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)n_f * n_t * npix;
  if (idx >= total) return;
  const int p = (int)(idx % npix);
  const long long r = idx / npix;
  const int t = (int)(r % n_t), f = (int)(r / n_t);
  const float m = mask[(mask_per_f ? (long long)f * npix : 0) + p];
  const float v = img[idx] * m;
  const long long o = ((long long)t * cube_f_total + cube_f0 + f) * npix + p;
  if (OUT_F16)
    reinterpret_cast<__half*>(cube)[o] = __float2half_rn(v);
  else
    reinterpret_cast<float*>(cube)[o] = v;
}

// ===========================================================================
// Compact-layout combine (combine_sparse_v4 + build_sparse_cell_csr,
// image/tiled_combine_cuda.py:966-1060, 1092-1240): streams in the
// time-minor compact layout dense[g][k][t][re, im] int8 (k a pattern cell of
// stream g), a CSR over the active half cells (u, w <= N/2) listing every
// stream g that carries the cell (k) or its mirror (km), -1 where absent.
// out[f][out_row0 + t][u][w] = 0.5 (sum_g q(k) + conj q(km)) at stream time
// t + t_lo - shift[f][g] (zero outside [0, t_rows)), times (-1)^(u+w) when
// fftshift; int32 sums, so exact; fp16 pairs or complex64.  Only active
// cells are written.
// One CTA per (active cell, tile of CS_T output times): the cell's entries
// go to shared memory, then each thread takes (fine DM, time) pairs; a
// warp's consecutive times read consecutive 2-byte stream words.
// ===========================================================================
constexpr int CS_T = 64;
constexpr int CS_MAXE = 64;

template <bool OUT_F16>
__global__ void __launch_bounds__(256) combine_sparse_kernel(
    const int16_t* __restrict__ dense, const int* __restrict__ cell_uw,
    const int* __restrict__ cell_ptr, const int* __restrict__ ent_g,
    const int* __restrict__ ent_k, const int* __restrict__ ent_km,
    const int* __restrict__ shifts, void* __restrict__ out, int n_sb, int t_rows, int t_pad,
    int nfm, int N, int n_fdm, int t_out_len, int t_lo, int fftshift, int out_rows,
    int out_row0, int* __restrict__ status) {
  __shared__ int s_g[CS_MAXE], s_k[CS_MAXE], s_km[CS_MAXE];
  const int a = blockIdx.x;
  const int nh = N / 2 + 1;
  const int uw = cell_uw[a];
  const int u = uw / nh, w = uw % nh;
  const int e0 = cell_ptr[a];
  const int ne = cell_ptr[a + 1] - e0;
  if (ne > CS_MAXE || ne < 0) {
    if (threadIdx.x == 0) dsb_flag(status, DSB_E_CAPACITY);
    return;
  }
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    const int g = ent_g[e0 + e], k = ent_k[e0 + e], km = ent_km[e0 + e];
    const bool ok = g >= 0 && g < n_sb && k < nfm && km < nfm;
    s_g[e] = ok ? g : -1;
    s_k[e] = k;
    s_km[e] = km;
    if (!ok) dsb_flag(status, DSB_E_ARG);
  }
  __syncthreads();
  const bool flip = fftshift && ((u + w) & 1);
  const int t0 = blockIdx.y * CS_T;
  const int nt = min(CS_T, t_out_len - t0);
  for (int idx = threadIdx.x; idx < n_fdm * CS_T; idx += blockDim.x) {
    const int f = idx / CS_T, tl = idx % CS_T;
    if (tl >= nt) continue;
    const int t = t0 + tl;
    int re = 0, im = 0;
    for (int e = 0; e < ne; ++e) {
      const int g = s_g[e];
      if (g < 0) continue;
      const int ts = t + t_lo - shifts[f * n_sb + g];
      if (ts < 0 || ts >= t_rows) continue;
      const long long row = (long long)g * nfm;
      if (s_k[e] >= 0) {
        const int16_t v = __ldg(dense + (row + s_k[e]) * t_pad + ts);
        re += (int)(int8_t)(v & 0xff);
        im += (int)(int8_t)((v >> 8) & 0xff);
      }
      if (s_km[e] >= 0) {
        const int16_t v = __ldg(dense + (row + s_km[e]) * t_pad + ts);
        re += (int)(int8_t)(v & 0xff);
        im -= (int)(int8_t)((v >> 8) & 0xff);
      }
    }
    float o_re = 0.5f * (float)re, o_im = 0.5f * (float)im;
    if (flip) {
      o_re = -o_re;
      o_im = -o_im;
    }
    const long long o = ((long long)f * out_rows + out_row0 + t) * N * nh + (long long)u * nh + w;
    if (OUT_F16)
      reinterpret_cast<__half2*>(out)[o] = __floats2half2_rn(o_re, o_im);
    else
      reinterpret_cast<float2*>(out)[o] = make_float2(o_re, o_im);
  }
}

// ===========================================================================
// padded cumsum / boxcars (detector/forward.py:250-455,
// detector/triton_boxcar.py:47-360).  Each prefix is accumulated in float64
// and rounded once to float32.
// ===========================================================================
template <typename T>
DSB_DEV float ldf(const T* p, long long i);
template <>
DSB_DEV float ldf<float>(const float* p, long long i) { return p[i]; }
template <>
DSB_DEV float ldf<__half>(const __half* p, long long i) { return __half2float(p[i]); }

template <typename T>
__global__ void padded_cumsum_kernel(const T* __restrict__ x, int n, long long inner, int max_w,
                                     float* __restrict__ cs) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= inner) return;
  const int pl = max_w / 2, pr = max_w - 1 - pl;
  for (int j = 0; j <= pl; ++j) cs[(long long)j * inner + e] = 0.f;
  double run = 0.0;
  float last = 0.f;
  for (int i = 0; i < n; ++i) {
    run += (double)ldf<T>(x, (long long)i * inner + e);
    last = (float)run;
    cs[(long long)(1 + pl + i) * inner + e] = last;
  }
  for (int r = 0; r < pr; ++r) cs[(long long)(1 + pl + n + r) * inner + e] = last;
}

// CHECK: every prefix row read must lie in [0, cs_rows); an output whose
// widths / offsets would read outside gets S/N NaN and winner -1 instead
// (the rows outside belong to no call's data: the shared scratch array of
// dsb_boxcar_argmax_noalloc).
template <bool OUT_F16, bool CHECK = false>
__global__ void multi_boxcar_argmax_kernel(const float* __restrict__ cs, long long inner,
                                           const int* __restrict__ widths,
                                           const int* __restrict__ offsets,
                                           const float* __restrict__ sinv, int K, int n_out,
                                           int t_base, void* __restrict__ out_max,
                                           int16_t* __restrict__ out_win, long long cs_rows = 0) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_out * inner) return;
  const int t = (int)(idx / inner);
  const long long e = idx % inner;
  const int ta = t + t_base;
  float best = 0.f;
  int win = 0;
  for (int k = 0; k < K; ++k) {
    const long long lo = (long long)ta + offsets[k], hi = lo + widths[k];
    if (CHECK && (lo < 0 || hi < 0 || lo >= cs_rows || hi >= cs_rows)) {
      best = __int_as_float(0x7fc00000);
      win = -1;
      break;
    }
    const float s = (cs[hi * inner + e] - cs[lo * inner + e]) * sinv[k];
    if (k == 0 || s > best) {
      best = s;
      win = k;
    }
  }
  if (OUT_F16)
    reinterpret_cast<__half*>(out_max)[idx] = __float2half_rn(best);
  else
    reinterpret_cast<float*>(out_max)[idx] = best;
  out_win[idx] = (int16_t)win;
}

__global__ void boxcar_from_cs_kernel(const float* __restrict__ cs, long long inner, int width,
                                      int start, int n_out, float* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_out * inner) return;
  const int t = (int)(idx / inner);
  const long long e = idx % inner;
  out[idx] = cs[(long long)(start + t + width) * inner + e] - cs[(long long)(start + t) * inner + e];
}

// ===========================================================================
// Fused streaming detector: per pixel, float64 running prefix rounded to
// float32 (identical to the padded cumsum above), a register ring of the
// last MAXW+1 prefixes, boxcar widths 1, 2, 4, ..., MAXW (centred, offsets
// MAXW/2 - w/2), S/N = (hi - lo) * sinv[k], strict '>' over k, and
// compaction of every output cell above threshold.
// ===========================================================================
struct DetCand {
  int t;      // output index (t_abs - t_base)
  int pix;    // (f * H + h) * W + w inside the cube
  float snr;
  int k;
};

// Element e = f * npix + p of time t is read at x[f*f_stride + t*t_stride + p]
// and multiplied by mask[f*npix + p] when a mask is given (the per-fine-DM
// edge mask x 1/sigma), so the detector consumes the FFT output directly.
// Layer-2 score samples (noise_norm/layer2.py, the streaming detector's
// per-kernel subsample, detector/forward.py:1425-1530): entries {eg, t, k,
// slot} sorted by (eg, t), eg = e + pix_off the cell's index over all fine
// DMs, t the output index (ta - t_base); off[gb] the first entry of global
// 256-cell block gb.  Each entry's raw boxcar sum of width 2^k (before the
// 1/sigma_k scale) goes to out[k * m + slot].  out == null: no sampling.
struct L2Samples {
  const int* off;
  const int4* ent;
  float* out;
  int m;
};

// The K boxcar sums (widths 1, 2, ..., 2^(K-1)) of one output, before the
// 1/sigma_k scale.
template <int K>
struct BoxSums {
  float v[K];
};

// Saturation level of the detector's candidate count (capacities are below it).
constexpr int DET_COUNT_MAX = 1 << 30;

// Exact strict-'>' winner over the widths (the lowest k wins ties) and, when
// its S/N passes thr, one appended candidate.  Out of line: called only for
// outputs the screen lets through.
template <int K>
__device__ __noinline__ void det_emit(const BoxSums<K> d, const float* __restrict__ sinv,
                                      float thr, int t_out, int pix,
                                      DetCand* __restrict__ cands, int cap,
                                      int* __restrict__ count) {
  float best = 0.f;
  int win = 0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float s = d.v[k] * __ldg(sinv + k);
    if (k == 0 || s > best) {
      best = s;
      win = k;
    }
  }
  if (best > thr) {
    // count[0] stops growing near DET_COUNT_MAX (above any capacity) instead
    // of wrapping to negative slots when nearly every cell passes: once the
    // buffer is full only the count's current value is read, and it is
    // raised while below the saturation level (concurrent raises overshoot
    // it by at most the resident threads)
    int slot = __ldcg(count);
    if (slot < cap)
      slot = atomicAdd(count, 1);
    else if (slot < DET_COUNT_MAX)
      atomicAdd(count, 1);
    if (slot < cap)
      cands[slot] = DetCand{t_out, pix, best, win};
    else  // the largest S/N that did not fit (positive floats order as ints)
      atomicMax(count + 1, __float_as_int(best));
  }
}

// Every Layer-2 entry of (cell eg, output t_out) from entry s_i on: the raw
// boxcar of its width into its slot.  Returns the next entry and its output
// time (0x7fffffff when this cell has no more).
template <int K>
__device__ __noinline__ int2 det_sample(const BoxSums<K> d, const L2Samples l2, int s_i,
                                        int s_end, int eg, int t_out) {
  int s_t = t_out;
  while (s_t == t_out) {
    const int4 en = __ldg(&l2.ent[s_i]);
    float v = 0.f;
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k == en.z) v = d.v[k];
    l2.out[(long long)en.z * l2.m + en.w] = v;
    ++s_i;
    s_t = (s_i < s_end && __ldg(&l2.ent[s_i].x) == eg) ? __ldg(&l2.ent[s_i].y) : 0x7fffffff;
  }
  return make_int2(s_i, s_t);
}

// One thread per cell; it marches the cell's time series once, keeping its
// last MAXW + 1 prefix sums in a register ring.  Time is walked in blocks of
// DB steps (unrolled; det_db): step j of a block writes its prefix to ring slot
// MAXW + j, and the block ends by moving the newest MAXW prefixes down to
// slots 0 .. MAXW-1 (MAXW register moves per DB steps), so the ring indices
// are compile-time constants while the unrolled code stays DB steps long.
// The inputs are prefetched DB steps ahead, one load per step.
// Boxcars to 32 or 64 (MAXW 32, 64): DB = 16 steps per block, inputs
// prefetched DP = 8 steps ahead (a rolling set of DP registers), so that ring
// and prefetch fit 128 registers: two CTAs per SM.  Narrower boxcars keep a
// short ring and run more CTAs per SM (three at 16: 80 registers, 16 steps
// per block; four below: 64 registers, 8 steps per block, 4 ahead), whose
// occupancy hides load latency better (at b16: 116 -> 96 ms per block of the
// 512-DM 256^2 workload against two CTAs per SM).
template <int LOGW>
struct DetCfg {
  // steps per block, prefetch depth, CTAs per SM (64 / 80 / 128 registers)
  static constexpr int DB = LOGW >= 4 ? 16 : 8;
  static constexpr int DP = LOGW >= 4 ? 8 : 4;
  static constexpr int MINB = LOGW >= 5 ? 2 : (LOGW == 4 ? 3 : 4);
};
constexpr int DET_PF = 32;  // L2 prefetch distance (steps)

DSB_DEV void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <int LOGW, typename T>
__global__ void __launch_bounds__(256, DetCfg<LOGW>::MINB) detect_kernel(const T* __restrict__ x, int n, int npix,
                                                     long long inner, long long f_stride,
                                                     long long t_stride,
                                                     const float* __restrict__ mask,
                                                     long long mask_f_stride,
                                                     const float* __restrict__ sig_f,
                                                     const float* __restrict__ sinv,
                                                     int t_base, int n_out, float thr,
                                                     DetCand* __restrict__ cands, int cap, int pix_off,
                                                     int* __restrict__ count, const L2Samples l2) {
  constexpr int MAXW = 1 << LOGW;
  constexpr int K = LOGW + 1;
  constexpr int PL = MAXW / 2;
  constexpr int DB = DetCfg<LOGW>::DB, DP = DetCfg<LOGW>::DP;
  constexpr int RS = MAXW + DB;  // ring registers
  static_assert(DB % DP == 0, "the prefetch set cycles within a block");
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= inner) return;
  // this cell's Layer-2 sample entries [s_i, s_end) (a few thousand per
  // kernel over the whole cube), s_t the output index of the next one
  int s_i = 0, s_end = 0, s_t = 0x7fffffff;
  const int eg = (int)e + pix_off;
  if (l2.out) {
    const int gb = pix_off / 256 + (int)blockIdx.x;
    int lo = __ldg(l2.off + gb);
    s_end = __ldg(l2.off + gb + 1);
    while (lo < s_end && __ldg(&l2.ent[lo].x) < eg) ++lo;
    s_i = lo;
    if (s_i < s_end && __ldg(&l2.ent[s_i].x) == eg) s_t = __ldg(&l2.ent[s_i].y);
  }
  const long long fidx = e / npix, p = e % npix;
  const T* cube = x + fidx * f_stride + p;
  // x * 1.0f == x exactly, so an absent mask costs one exact multiply
  float mval = mask ? mask[fidx * mask_f_stride + p] : 1.0f;
  if (sig_f) mval = mval / sig_f[fidx];
  float tau[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    // screen level of width k: a boxcar sum d can give fl(d * si) > thr only
    // if d > thr / si up to two roundings (2^-23 relative), so a level
    // lowered by 2^-20 of its magnitude never misses one
    const float lv = thr / sinv[k];
    tau[k] = lv - fabsf(lv) * 0x1p-20f;
  }
  // ring[i] holds prefix J0 - MAXW + i at the start of the block of steps
  // J0 .. J0 + DB - 1 (prefix index J: 0 for J <= PL, the running sum of
  // inputs 0 .. J-PL-1 up to J = PL + n, then the last sum: the padded
  // cumsum); the output of step J is ta = J - MAXW and reads ring slots
  // j .. j + MAXW
  float ring[RS];
#pragma unroll
  for (int q = 0; q < RS; ++q) ring[q] = 0.f;
  double run = 0.0;
  float last = 0.f;
  const int total = n + MAXW;  // cs length
  // One output: the screen compares each boxcar sum with its lowered level
  // (a superset of what the exact strict-'>' chain of det_emit reports,
  // which decides); the threshold hits and the Layer-2 samples are rare, so
  // both are calls out of the unrolled loop.
  auto output = [&](int j, int ta, auto with_samples) {
    BoxSums<K> d;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int w = 1 << k;
      const int off = PL - w / 2;
      d.v[k] = ring[j + off + w] - ring[j + off];
    }
    bool hit = false;
#pragma unroll
    for (int k = 0; k < K; ++k) hit |= d.v[k] > tau[k];
    if (hit) det_emit<K>(d, sinv, thr, ta - t_base, (int)e + pix_off, cands, cap, count);
    if (decltype(with_samples)::value && ta - t_base == s_t) {
      const int2 r = det_sample<K>(d, l2, s_i, s_end, eg, ta - t_base);
      s_i = r.x;
      s_t = r.y;
    }
  };
  // input of step J: x[J - 1 - PL] (for PL < J <= PL + n); xin[j % DP]
  // holds the input of step J0 + j, loaded DP steps earlier
  auto input = [&](int J) -> float {
    const int i = J - 1 - PL;
    return (i >= 0 && i < n) ? ldf<T>(cube, (long long)i * t_stride) : 0.f;
  };
  float xin[DP];
#pragma unroll
  for (int j = 0; j < DP; ++j) xin[j] = input(j);
  // the first steps produce no output (ta < t_base): prefixes only
  const int warm_end = t_base + MAXW;
  // blocks after the last output step (J = t_base + n_out - 1 + MAXW) feed
  // nothing: the cell is done
  const int out_end = t_base + n_out + MAXW;
  for (int J0 = 0; J0 < total && J0 < out_end; J0 += DB) {
    if (J0 + DB <= warm_end && J0 + DB + DP - 1 - PL <= n) {
#pragma unroll
      for (int j = 0; j < DB; ++j) {
        const int J = J0 + j;
        float v = 0.f;
        if (J > PL) {
          run += (double)(xin[j % DP] * mval);
          v = (float)run;
        }
        ring[MAXW + j] = v;
        xin[j % DP] = input(J + DP);
      }
      last = ring[MAXW + DB - 1];
    } else if (J0 >= PL + 1 && J0 + DB - 1 <= PL + n && J0 - MAXW >= t_base &&
               J0 + DB - 1 - MAXW < t_base + n_out && J0 + DB - 1 + DP - 1 - PL < n) {
      // steady state: every step an input, a prefix and an output, and the
      // prefetched input in range; the Layer-2 test only in the (rare)
      // blocks that hold this cell's next sample
      const T* nxt = cube + (long long)(J0 + DP - 1 - PL) * t_stride;
      // L2 prefetch DET_PF steps ahead, the block's DB lines in one
      // instruction: lane j < DB takes step J0 + j's line of the warp (lane
      // 0's cell), where still inside the cube
      // (lane 0's cell is always active when any lane of its warp is; the
      // branch is warp-uniform, so the warp's live lanes are all here)
      {
        const unsigned lane = threadIdx.x & 31;
        const long long n_live = inner - (e - lane);  // lanes of this warp with a cell
        const unsigned live = n_live >= 32 ? 0xffffffffu : ((1u << n_live) - 1u);
        const T* cube0 = reinterpret_cast<const T*>(
            __shfl_sync(live, reinterpret_cast<unsigned long long>(cube), 0));
        const int ipf = J0 + (int)lane + DET_PF - 1 - PL;
        if (lane < (unsigned)DB && ipf < n) prefetch_l2(cube0 + (long long)ipf * t_stride);
      }
      auto steady = [&](auto with_samples) {
#pragma unroll
        for (int j = 0; j < DB; ++j) {
          run += (double)(xin[j % DP] * mval);
          ring[MAXW + j] = (float)run;
          xin[j % DP] = ldf<T>(nxt, (long long)j * t_stride);
          output(j, J0 + j - MAXW, with_samples);
        }
      };
      if ((unsigned)(s_t - (J0 - MAXW - t_base)) < (unsigned)DB)
        steady(std::true_type{});
      else
        steady(std::false_type{});
      last = ring[MAXW + DB - 1];
    } else {
#pragma unroll
      for (int j = 0; j < DB; ++j) {
        const int J = J0 + j;
        if (J < total) {
          float v;
          if (J <= PL) {
            v = 0.f;
          } else if (J <= PL + n) {
            run += (double)(xin[j % DP] * mval);
            last = (float)run;
            v = last;
          } else {
            v = last;
          }
          ring[MAXW + j] = v;
          const int ta = J - MAXW;
          if (ta >= t_base && ta < t_base + n_out) output(j, ta, std::true_type{});
        }
        xin[j % DP] = input(J + DP);
      }
    }
#pragma unroll
    for (int q = 0; q < MAXW; ++q) ring[q] = ring[q + DB];
  }
}

// The same detector with the cube staged in shared memory by TMA (float
// cubes whose fine DMs are whole warps of cells: npix a multiple of 32).
// Each warp owns 32 consecutive cells of one fine DM and a ring of NST
// shared-memory stages, each one block of DB times x 32 cells (one 3-D tile
// of the cube's tensor map, completing on the stage's mbarrier).  Lane 0
// issues block b + NST - 1 when the warp starts block b, so the copies
// run NST - 1 blocks ahead with no registers held for them and no barrier
// wider than the warp; times outside [0, n) arrive as zeros.  The marching,
// the screen and the rare paths are detect_kernel's, so the outputs are the
// same bits.  A wait that does not complete within DSB_SPIN_LIMIT polls sets
// count[1] to a quiet NaN (DET_TIMEOUT_BITS) and ends the warp after waiting,
// again bounded, for its copies in flight.
constexpr int DET_TIMEOUT_BITS = 0x7fc00000;

// Steps per block and stages of the TMA form: with the inputs out of the
// registers, boxcars to 64 afford 32-step blocks (96 ring registers, half
// the ring moves per step) in three stages of 4 KB per warp; the narrower
// widths keep detect_kernel's blocks in four stages.
template <int LOGW>
struct DetTmaCfg {
  static constexpr int DB = LOGW == 6 ? 32 : DetCfg<LOGW>::DB;
  static constexpr int NST = LOGW == 6 ? 3 : 4;
};

template <int LOGW>
constexpr int det_tma_smem() {
  return 8 * DetTmaCfg<LOGW>::NST * DetTmaCfg<LOGW>::DB * 32 * 4 + 8 * DetTmaCfg<LOGW>::NST * 8;
}

template <int LOGW>
__global__ void __launch_bounds__(256, DetCfg<LOGW>::MINB)
    detect_tma_kernel(const __grid_constant__ CUtensorMap tmap, int n, int npix, long long inner,
                      const float* __restrict__ mask, long long mask_f_stride,
                      const float* __restrict__ sig_f, const float* __restrict__ sinv,
                      int t_base, int n_out, float thr, DetCand* __restrict__ cands, int cap,
                      int pix_off, int* __restrict__ count, const L2Samples l2) {
  constexpr int MAXW = 1 << LOGW;
  constexpr int K = LOGW + 1;
  constexpr int PL = MAXW / 2;
  constexpr int DB = DetTmaCfg<LOGW>::DB;
  constexpr int DET_NST = DetTmaCfg<LOGW>::NST;
  constexpr int RS = MAXW + DB;  // ring registers
  constexpr int SB = DB * 32;    // floats per stage
  extern __shared__ __align__(128) uint8_t det_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* stages = reinterpret_cast<float*>(det_smem) + warp * DET_NST * SB;
  uint64_t* bars = reinterpret_cast<uint64_t*>(det_smem + 8 * DET_NST * SB * 4) + warp * DET_NST;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // npix % 32 == 0, so inner is whole warps: a warp is in or out as a whole
  if (e >= inner) return;
  int s_i = 0, s_end = 0, s_t = 0x7fffffff;
  const int eg = (int)e + pix_off;
  if (l2.out) {
    const int gb = pix_off / 256 + (int)blockIdx.x;
    int lo = __ldg(l2.off + gb);
    s_end = __ldg(l2.off + gb + 1);
    while (lo < s_end && __ldg(&l2.ent[lo].x) < eg) ++lo;
    s_i = lo;
    if (s_i < s_end && __ldg(&l2.ent[s_i].x) == eg) s_t = __ldg(&l2.ent[s_i].y);
  }
  const long long fidx = e / npix, p = e % npix;
  const int p0 = (int)(p - lane);  // the warp's first cell (a multiple of 32)
  float mval = mask ? mask[fidx * mask_f_stride + p] : 1.0f;
  if (sig_f) mval = mval / sig_f[fidx];
  float tau[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const float lv = thr / sinv[k];
    tau[k] = lv - fabsf(lv) * 0x1p-20f;
  }
  // the ring as float32 pairs (slot i in rg[i / 2], .x even, .y odd), so
  // that two consecutive steps' boxcars of one width are one packed
  // float32x2 subtraction where their slots align (widths 4 and up)
  float2 rg[(RS + 1) / 2];
#pragma unroll
  for (int q = 0; q < (RS + 1) / 2; ++q) rg[q] = make_float2(0.f, 0.f);
  auto ring = [&](int i) -> float& { return (i & 1) ? rg[i >> 1].y : rg[i >> 1].x; };
  double run = 0.0;
  float last = 0.f;
  const int total = n + MAXW;
  const int warm_end = t_base + MAXW;
  const int out_end = t_base + n_out + MAXW;
  const int n_blk = (min(total, out_end) + DB - 1) / DB;
  // block b holds inputs x[b DB - 1 - PL .. b DB + DB - 2 - PL]; a block with
  // none inside the cube completes its phase with no copy (its inputs are
  // never read)
  auto issue = [&](int b) {
    uint64_t* bar = bars + b % DET_NST;
    const int y0 = b * DB - 1 - PL;
    if (y0 < n && y0 + DB > 0) {
      mbar_arrive_expect_tx(bar, SB * 4);
      tma_load_3d(stages + (b % DET_NST) * SB, &tmap, p0, y0, (int)fidx, bar);
    } else {
      mbar_arrive(bar);
    }
  };
  if (lane == 0) {
    for (int s = 0; s < DET_NST; ++s) mbar_init(bars + s, 1);
    fence_mbar_init();
    for (int b = 0; b < min(DET_NST - 1, n_blk); ++b) issue(b);
  }
  __syncwarp();
  // the screen, the threshold hits and the Layer-2 samples of one output
  // from its boxcar sums
  auto decide = [&](const BoxSums<K>& d, int ta, auto with_samples) {
    bool hit = false;
#pragma unroll
    for (int k = 0; k < K; ++k) hit |= d.v[k] > tau[k];
    if (hit) det_emit<K>(d, sinv, thr, ta - t_base, (int)e + pix_off, cands, cap, count);
    if (decltype(with_samples)::value && ta - t_base == s_t) {
      const int2 r = det_sample<K>(d, l2, s_i, s_end, eg, ta - t_base);
      s_i = r.x;
      s_t = r.y;
    }
  };
  auto output = [&](int j, int ta, auto with_samples) {
    BoxSums<K> d;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int w = 1 << k;
      const int off = PL - w / 2;
      d.v[k] = ring(j + off + w) - ring(j + off);
    }
    decide(d, ta, with_samples);
  };
  // the screens of steps j and j + 1 (j even): widths 1 and 2 one by one,
  // the wider ones (both slots even) as packed pairs, with the same
  // roundings; an output that passes a screen or holds a Layer-2 sample
  // (rare) recomputes its sums from the ring and decides as output does
  auto output2 = [&](int j, int ta, auto with_samples) {
    bool hit0 = false, hit1 = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int w = 1 << k;
      const int off = PL - w / 2;
      if (w >= 4 && PL % 2 == 0) {
        const float2 dd = f2_sub(rg[(j + off + w) >> 1], rg[(j + off) >> 1]);
        hit0 |= dd.x > tau[k];
        hit1 |= dd.y > tau[k];
      } else {
        hit0 |= ring(j + off + w) - ring(j + off) > tau[k];
        hit1 |= ring(j + 1 + off + w) - ring(j + 1 + off) > tau[k];
      }
    }
    if (hit0 || (decltype(with_samples)::value && ta - t_base == s_t))
      output(j, ta, with_samples);
    if (hit1 || (decltype(with_samples)::value && ta + 1 - t_base == s_t))
      output(j + 1, ta + 1, with_samples);
  };
  int b = 0;
  bool ok = true;
  for (; b < n_blk; ++b) {
    const int J0 = b * DB;
    // every lane is done with block b - 1, whose stage takes block
    // b + DET_NST - 1 (generic-proxy reads before the async-proxy write)
    __syncwarp();
    if (lane == 0 && b + DET_NST - 1 < n_blk) {
      fence_proxy_async_smem();
      issue(b + DET_NST - 1);
    }
    if (!__all_sync(0xffffffffu,
                    mbar_wait(bars + b % DET_NST, (uint32_t)((b / DET_NST) & 1)))) {
      ok = false;
      break;
    }
    // input of step J0 + j (x[J0 + j - 1 - PL]) at sx[32 j]
    const float* sx = stages + (b % DET_NST) * SB + lane;
    if (J0 + DB <= warm_end && J0 + DB - 2 - PL < n) {
#pragma unroll
      for (int j = 0; j < DB; ++j) {
        const int J = J0 + j;
        float v = 0.f;
        if (J > PL) {
          run += (double)(sx[32 * j] * mval);
          v = (float)run;
        }
        ring(MAXW + j) = v;
      }
      last = ring(MAXW + DB - 1);
    } else if (J0 >= PL + 1 && J0 + DB - 1 <= PL + n && J0 - MAXW >= t_base &&
               J0 + DB - 1 - MAXW < t_base + n_out) {
      auto steady = [&](auto with_samples) {
#pragma unroll
        for (int j = 0; j < DB; j += 2) {
          run += (double)(sx[32 * j] * mval);
          ring(MAXW + j) = (float)run;
          run += (double)(sx[32 * (j + 1)] * mval);
          ring(MAXW + j + 1) = (float)run;
          output2(j, J0 + j - MAXW, with_samples);
        }
      };
      if ((unsigned)(s_t - (J0 - MAXW - t_base)) < (unsigned)DB)
        steady(std::true_type{});
      else
        steady(std::false_type{});
      last = ring(MAXW + DB - 1);
    } else {
#pragma unroll
      for (int j = 0; j < DB; ++j) {
        const int J = J0 + j;
        if (J < total) {
          float v;
          if (J <= PL) {
            v = 0.f;
          } else if (J <= PL + n) {
            run += (double)(sx[32 * j] * mval);
            last = (float)run;
            v = last;
          } else {
            v = last;
          }
          ring(MAXW + j) = v;
          const int ta = J - MAXW;
          if (ta >= t_base && ta < t_base + n_out) output(j, ta, std::true_type{});
        }
      }
    }
    static_assert(DB % 2 == 0, "blocks of whole slot pairs");
#pragma unroll
    for (int q = 0; q < (MAXW + 1) / 2; ++q) rg[q] = rg[q + DB / 2];
  }
  if (!ok && lane == 0) {
    atomicMax(count + 1, DET_TIMEOUT_BITS);
    for (int c = b; c < min(n_blk, b + DET_NST); ++c)
      mbar_wait(bars + c % DET_NST, (uint32_t)((c / DET_NST) & 1));
  }
}

// ===========================================================================
// Layer-1 sigma-clipped std (noise_norm/layer1.py:53-125): one block per
// row, rows of at most L1_MAX samples; bitonic sort, then the clipping
// iterations walk a contiguous range of the sorted row; median is the lower
// median (torch.nanmedian); sums in float64.
// ===========================================================================
constexpr int L1_MAX = 4096;
constexpr int L1_THREADS = 1024;
static_assert(L1_MAX % L1_THREADS == 0, "each thread stages a whole number of samples");

// Where a row's samples come from: a [rows, m] matrix, or (GATHER) the
// images themselves, sample i of row f = img[f*f_stride + times[i / n_pix] *
// t_stride + pix[i % n_pix]] (the Layer-1 subsample of the pipeline).
struct L1Src {
  const float* x;
  long long f_stride, t_stride;
  const int* times;
  const int* pix;
  int n_pix;
  int nonpos_to_one;  // report sigma <= 0 (or NaN) as 1 (the mask divisor)
};

template <bool GATHER>
__global__ void __launch_bounds__(L1_THREADS) clipped_std_kernel(const L1Src src, int m,
                                                                 float n_sigma, int n_iter,
                                                                 float* __restrict__ out) {
  __shared__ __align__(16) float v[L1_MAX];
  __shared__ double red[L1_THREADS / 32];
  __shared__ int s_lo, s_hi;
  const float* row = src.x + (long long)blockIdx.x * (GATHER ? src.f_stride : m);
  int P = 1;
  while (P < m) P <<= 1;
  // Thread t holds samples 4t .. 4t + 3 in registers (every load issues
  // before the first is used); the padding past m is +inf.  The bitonic
  // network sorts all L1_MAX entries: its stages with partner distance j < 4
  // run inside the thread, 4 <= j <= 64 across the warp by shuffles, and only
  // j >= 128 through shared memory with a barrier (15 of the 78 stages).
  // The smallest P entries are the P entries of the P-padded sort, so the
  // result is the same as sorting P.
  static_assert(L1_MAX == 4 * L1_THREADS, "four samples per thread");
  float r[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = 4 * threadIdx.x + q;
    r[q] = __int_as_float(0x7f800000);
    if (i < m) {
      if constexpr (GATHER)
        r[q] = row[src.times[i / src.n_pix] * src.t_stride + src.pix[i % src.n_pix]];
      else
        r[q] = row[i];
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (!(r[q] == r[q]) || isinf(r[q])) r[q] = __int_as_float(0x7f800000);  // non-finite -> +inf
  const int i0 = 4 * threadIdx.x;
  float4* v4 = reinterpret_cast<float4*>(v);
  // compare-exchange of positions (i, i ^ j), i the lower: ascending where
  // (i & k) == 0
  auto cx = [](float& lo, float& hi, bool up) {
    if ((lo > hi) == up) {
      const float t = lo;
      lo = hi;
      hi = t;
    }
  };
  for (int k = 2; k <= L1_MAX; k <<= 1) {
    const bool up = (i0 & k) == 0;  // for k >= 4 the same for all four samples
    int j = k >> 1;
    if (j >= 128) {
      v4[threadIdx.x] = make_float4(r[0], r[1], r[2], r[3]);
      __syncthreads();
      for (; j >= 128; j >>= 1) {
        for (int i = threadIdx.x; i < L1_MAX; i += L1_THREADS) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const bool u = (i & k) == 0;
            const float a = v[i], b = v[ixj];
            if ((a > b) == u) {
              v[i] = b;
              v[ixj] = a;
            }
          }
        }
        __syncthreads();
      }
      const float4 w = v4[threadIdx.x];
      r[0] = w.x; r[1] = w.y; r[2] = w.z; r[3] = w.w;
    }
    for (; j >= 4; j >>= 1) {
      const bool lower = (i0 & j) == 0;  // this thread's samples are the lower positions
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float o = __shfl_xor_sync(0xffffffffu, r[q], j >> 2);
        // the lower position keeps the smaller value where ascending
        const bool keep_small = lower == up;
        r[q] = keep_small ? (o < r[q] ? o : r[q]) : (o > r[q] ? o : r[q]);
      }
    }
    if (k >= 4) {  // j = 2: pairs (0, 2), (1, 3)
      cx(r[0], r[2], up);
      cx(r[1], r[3], up);
    }
    {  // j = 1: pairs (0, 1), (2, 3); for k = 2 the direction alternates per pair
      cx(r[0], r[1], k == 2 ? ((i0 & 2) == 0) : up);
      cx(r[2], r[3], k == 2 ? (((i0 + 2) & 2) == 0) : up);
    }
  }
  v4[threadIdx.x] = make_float4(r[0], r[1], r[2], r[3]);
  __syncthreads();
  // finite count
  if (threadIdx.x == 0) {
    int n_fin = 0;
    int lo = 0, hi = P;
    while (lo < hi) {
      const int mid = (lo + hi) / 2;
      if (isinf(v[mid]) && v[mid] > 0) hi = mid; else lo = mid + 1;
    }
    n_fin = lo;
    s_lo = 0;
    s_hi = n_fin;
  }
  __syncthreads();
  float sigma = 0.f, med = 0.f;
  for (int it = 0; it <= n_iter; ++it) {
    const int lo = s_lo, hi = s_hi;
    const int cnt = hi - lo;
    if (cnt <= 0) {
      sigma = __int_as_float(0x7fc00000);
      break;
    }
    med = v[lo + (cnt - 1) / 2];
    double acc = 0.0;
    for (int i = lo + threadIdx.x; i < hi; i += L1_THREADS) {
      const float d = v[i] - med;
      acc += (double)(d * d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0.0;
      for (int w = 0; w < L1_THREADS / 32; ++w) tot += red[w];
      red[0] = tot;
    }
    __syncthreads();
    sigma = sqrtf((float)red[0] / (float)cnt);
    __syncthreads();
    if (it == n_iter) break;
    if (threadIdx.x == 0) {
      const float lo_v = med - n_sigma * sigma, hi_v = med + n_sigma * sigma;
      int a = lo, b = hi;
      while (a < hi && v[a] < lo_v) ++a;
      while (b > a && v[b - 1] > hi_v) --b;
      s_lo = a;
      s_hi = b;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    float o = (sigma == sigma) ? sigma : 0.f;
    if (src.nonpos_to_one && !(o > 0.f)) o = 1.f;
    out[blockIdx.x] = o;
  }
}

// The driver's tensor-map encoder, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 det_tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* q = nullptr;
    cudaDriverEntryPointQueryResult r;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &r) ==
            cudaSuccess &&
        r == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(q);
    cudaGetLastError();
  }
  return fn;
}

// The float cube as a 3-D tensor (cell, time, fine DM) with one detector
// block's box (32 cells x db times x 1).  False when the layout does not
// allow it (the caller then runs detect_kernel): npix a multiple of 32, the
// base 16-byte aligned, the strides whole 16-byte units.
bool det_cube_tmap(const float* x, int n, int n_f, int npix, long long f_stride,
                   long long t_stride, int db, CUtensorMap* m) {
  if (npix % 32 || (reinterpret_cast<uintptr_t>(x) & 15) || t_stride % 4 || t_stride < npix ||
      (n_f > 1 && (f_stride % 4 || f_stride < (long long)n * t_stride)))
    return false;
  auto fn = det_tmap_encoder();
  if (!fn) return false;
  const long long fs = n_f > 1 ? f_stride : (long long)n * t_stride;
  const cuuint64_t dims[3] = {(cuuint64_t)npix, (cuuint64_t)n, (cuuint64_t)n_f};
  const cuuint64_t strides[2] = {(cuuint64_t)t_stride * 4, (cuuint64_t)fs * 4};
  const cuuint32_t box[3] = {32u, (cuuint32_t)db, 1u};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(x), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int LOGW>
int det_tma_launch(const float* x, int n, int n_f, int npix, long long f_stride,
                   long long t_stride, const float* mask, long long mask_f_stride,
                   const float* sig_f, const float* sinv, int t_base, int n_out, float thr,
                   DetCand* c, int cap, int pix_off, int* count, const L2Samples& l2,
                   cudaStream_t stream, bool* done) {
  *done = false;
  CUtensorMap tm;
  memset(&tm, 0, sizeof(tm));
  if (!det_cube_tmap(x, n, n_f, npix, f_stride, t_stride, DetTmaCfg<LOGW>::DB, &tm))
    return DSB_OK;
  constexpr int smem = det_tma_smem<LOGW>();
  if (cudaFuncSetAttribute(detect_tma_kernel<LOGW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem) != cudaSuccess)
    return DSB_E_CUDA;
  const long long inner = (long long)n_f * npix;
  const unsigned grid = (unsigned)((inner + 255) / 256);
  detect_tma_kernel<LOGW><<<grid, 256, smem, stream>>>(tm, n, npix, inner, mask, mask_f_stride,
                                                       sig_f, sinv, t_base, n_out, thr, c, cap,
                                                       pix_off, count, l2);
  *done = true;
  return launch_status();
}

}  // namespace

extern "C" {

int dsb_uv_cells(const double* du, const double* dv, int n_bl, const double* nu_ghz, int n_ch,
                 double cell_lambda, int n_grid, int* row, int* col, cudaStream_t stream) {
  if (!du || !dv || !nu_ghz || !row || !col || n_bl < 0 || n_ch <= 0 || !(cell_lambda > 0))
    return DSB_E_ARG;
  const long long n = (long long)n_bl * n_ch;
  if (n == 0) return DSB_OK;
  uv_cells_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(du, dv, n_bl, nu_ghz, n_ch,
                                                                   cell_lambda, n_grid / 2, row,
                                                                   col);
  return launch_status();
}

int dsb_combine_rows(const void* D, int d_format, const long long* seg_base, const int* seg_depth,
                     const float* scales, const long long* sc_base, int n_coarse,
                     const int* hc_off, const int* e_g, const int* e_cell, const int* d_pitch,
                     const int* sfine, const int* f2c, int f0, int n_f, int G, int N,
                     long long t0, int n_t, int fftshift, void* out, cudaStream_t stream) {
  if (!D || !seg_base || !seg_depth || n_coarse <= 0 || !hc_off || !e_g || !e_cell ||
      !d_pitch || !sfine || !f2c || !out || d_format < 0 || d_format > 2 ||
      (d_format == 2 && (!scales || !sc_base)))
    return DSB_E_ARG;
  if (N <= 0 || (N & 1) || n_f <= 0 || n_t <= 0 || G <= 0) return DSB_E_ARG;
  CombArgs A{D, scales, sc_base, seg_base, seg_depth, n_coarse, hc_off, e_g, e_cell, d_pitch,
             sfine, f2c, f0, n_f, G, N, t0, n_t, fftshift, (float2*)out};
  const int n_hc = N * (N / 2 + 1);
  dim3 grid((n_hc + 127) / 128, n_f);
  if (d_format == 2)
    combine_rows_kernel<2><<<grid, 128, 0, stream>>>(A);
  else if (d_format == 1)
    combine_rows_kernel<1><<<grid, 128, 0, stream>>>(A);
  else
    combine_rows_kernel<0><<<grid, 128, 0, stream>>>(A);
  return launch_status();
}

int dsb_combine_sparse(const void* dense, const int* cell_uw, const int* cell_ptr,
                       const int* ent_g, const int* ent_k, const int* ent_km, int n_act,
                       const int* shifts, void* out, int out_f16, int n_sb, int t_rows,
                       int t_pad, int n_filled_max, int N, int n_fdm, int t_out_len, int t_lo,
                       int fftshift, int out_rows, int out_row0, int* status,
                       cudaStream_t stream) {
  if (!dense || !cell_uw || !cell_ptr || !shifts || !out || !status || n_act < 0 ||
      n_sb <= 0 || t_rows < 0 || t_pad < t_rows || n_filled_max <= 0 || N <= 0 || (N & 1) ||
      n_fdm <= 0 || t_out_len < 0 || out_row0 < 0 || out_row0 + t_out_len > out_rows)
    return DSB_E_ARG;
  if (n_act > 0 && (!ent_g || !ent_k || !ent_km)) return DSB_E_ARG;
  if ((reinterpret_cast<uintptr_t>(dense) & 1) || (reinterpret_cast<uintptr_t>(out) & 3))
    return DSB_E_ARG;
  if (n_act == 0 || t_out_len == 0) return DSB_OK;
  if ((t_out_len + CS_T - 1) / CS_T > 65535) return DSB_E_ARG;
  const dim3 grid(n_act, (t_out_len + CS_T - 1) / CS_T);
  if (out_f16)
    combine_sparse_kernel<true><<<grid, 256, 0, stream>>>(
        static_cast<const int16_t*>(dense), cell_uw, cell_ptr, ent_g, ent_k, ent_km, shifts, out,
        n_sb, t_rows, t_pad, n_filled_max, N, n_fdm, t_out_len, t_lo, fftshift, out_rows,
        out_row0, status);
  else
    combine_sparse_kernel<false><<<grid, 256, 0, stream>>>(
        static_cast<const int16_t*>(dense), cell_uw, cell_ptr, ent_g, ent_k, ent_km, shifts, out,
        n_sb, t_rows, t_pad, n_filled_max, N, n_fdm, t_out_len, t_lo, fftshift, out_rows,
        out_row0, status);
  return launch_status();
}

int dsb_combine_dense(const void* streams, const int* shifts, const float* scales,
                      const float* off_re, const float* off_im, int per_t, void* out,
                      int out_f16, int half,
                      int G, int t_stream, int t_det, int N, int t_lo, int fftshift,
                      cudaStream_t stream) {
  if (!streams || !shifts || !out || G <= 0 || N <= 0 || t_det <= t_lo || t_lo < 0) return DSB_E_ARG;
  if (half && (N & 1)) return DSB_E_ARG;
  const bool calib = scales != nullptr;
  if (calib && (!off_re || !off_im)) return DSB_E_ARG;
  const int nw = half ? N / 2 + 1 : N;
  dim3 block(32, 4, 8);
  dim3 grid((nw + 31) / 32, (N + 3) / 4, (t_det - t_lo + 7) / 8);
  const int8_t* s = (const int8_t*)streams;
  auto go = [&](auto h, auto c, auto f, auto pt) {
    combine_dense_kernel<decltype(h)::value, decltype(c)::value, decltype(f)::value,
                         decltype(pt)::value><<<grid, block, 0, stream>>>(
        s, shifts, scales, off_re, off_im, out, G, t_stream, t_det, N, t_lo, fftshift);
  };
  using T = std::true_type;
  using F = std::false_type;
  auto by_f = [&](auto h, auto c, auto pt) { out_f16 ? go(h, c, T{}, pt) : go(h, c, F{}, pt); };
  auto by_c = [&](auto h) {
    if (!calib) by_f(h, F{}, F{});
    else if (per_t) by_f(h, T{}, T{});
    else by_f(h, T{}, F{});
  };
  half ? by_c(T{}) : by_c(F{});
  return launch_status();
}

int dsb_mask_to_cube(const float* img, const float* mask, int mask_per_f, int n_f, int n_t,
                     int npix, void* cube, int cube_f16, int cube_f_total, int cube_f0,
                     cudaStream_t stream) {
  if (!img || !mask || !cube || n_f <= 0 || n_t <= 0 || npix <= 0) return DSB_E_ARG;
  if (cube_f0 < 0 || cube_f0 + n_f > cube_f_total) return DSB_E_ARG;
  const long long total = (long long)n_f * n_t * npix;
  if (cube_f16)
    mask_to_cube_kernel<true><<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(
        img, mask, mask_per_f, n_f, n_t, npix, cube, cube_f_total, cube_f0);
  else
    mask_to_cube_kernel<false><<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(
        img, mask, mask_per_f, n_f, n_t, npix, cube, cube_f_total, cube_f0);
  return launch_status();
}

int dsb_padded_cumsum(const void* x, int x_f16, int n, long long inner, int max_w, float* cs,
                      cudaStream_t stream) {
  if (!x || !cs || n <= 0 || inner <= 0 || max_w < 1 || max_w > n) return DSB_E_ARG;
  const unsigned grid = (unsigned)((inner + 255) / 256);
  if (x_f16)
    padded_cumsum_kernel<__half><<<grid, 256, 0, stream>>>((const __half*)x, n, inner, max_w, cs);
  else
    padded_cumsum_kernel<float><<<grid, 256, 0, stream>>>((const float*)x, n, inner, max_w, cs);
  return launch_status();
}

int dsb_multi_boxcar_argmax(const float* cs, long long inner, const int* widths,
                            const int* offsets, const float* sigma_inv, int K, int n_out,
                            int t_base, void* out_max, int out_f16, void* out_win,
                            cudaStream_t stream) {
  if (!cs || !widths || !offsets || !sigma_inv || !out_max || !out_win || K < 1 || n_out <= 0)
    return DSB_E_ARG;
  const long long total = (long long)n_out * inner;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (out_f16)
    multi_boxcar_argmax_kernel<true><<<grid, 256, 0, stream>>>(
        cs, inner, widths, offsets, sigma_inv, K, n_out, t_base, out_max, (int16_t*)out_win);
  else
    multi_boxcar_argmax_kernel<false><<<grid, 256, 0, stream>>>(
        cs, inner, widths, offsets, sigma_inv, K, n_out, t_base, out_max, (int16_t*)out_win);
  return launch_status();
}

int dsb_boxcar_from_cs(const float* cs, long long inner, int width, int start, int n_out,
                       float* out, cudaStream_t stream) {
  if (!cs || !out || width < 1 || start < 0 || n_out <= 0) return DSB_E_ARG;
  const long long total = (long long)n_out * inner;
  boxcar_from_cs_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(cs, inner, width,
                                                                             start, n_out, out);
  return launch_status();
}

int dsb_detect(const void* cube, int cube_f16, int n, int n_f, int npix, long long f_stride,
               long long t_stride, const float* mask, long long mask_f_stride,
               const float* sig_f, int log_maxw, const float* sigma_inv,
               int t_base, int n_out, float threshold, void* cands, int cap, int pix_off,
               int* count, cudaStream_t stream) {
  return dsb_detect_sampled(cube, cube_f16, n, n_f, npix, f_stride, t_stride, mask,
                            mask_f_stride, sig_f, log_maxw, sigma_inv, t_base, n_out, threshold,
                            cands, cap, pix_off, count, nullptr, nullptr, nullptr, 0, stream);
}

int dsb_detect_sampled(const void* cube, int cube_f16, int n, int n_f, int npix,
                       long long f_stride, long long t_stride, const float* mask,
                       long long mask_f_stride, const float* sig_f, int log_maxw,
                       const float* sigma_inv, int t_base, int n_out, float threshold,
                       void* cands, int cap, int pix_off, int* count, const int* l2_off,
                       const void* l2_ent, float* l2_out, int l2_m, cudaStream_t stream) {
  if (!cube || !sigma_inv || !cands || !count || n <= 0 || n_f <= 0 || npix <= 0 || cap < 0 ||
      cap > DET_COUNT_MAX)
    return DSB_E_ARG;
  if (l2_out && (!l2_off || !l2_ent || l2_m <= 0 || pix_off < 0 || (pix_off % 256) != 0 ||
                 (reinterpret_cast<uintptr_t>(l2_ent) & 15)))
    return DSB_E_ARG;
  if ((long long)n_f * npix + pix_off > 0x7fffffffLL) return DSB_E_ARG;
  const L2Samples l2{l2_off, static_cast<const int4*>(l2_ent), l2_out, l2_m};
  if (log_maxw < 0 || log_maxw > 6 || (1 << log_maxw) > n || t_base < 0 || n_out < 0 ||
      t_base + n_out > n)
    return DSB_E_ARG;
  const long long inner = (long long)n_f * npix;
  const unsigned grid = (unsigned)((inner + 255) / 256);
  DetCand* c = (DetCand*)cands;
  if (!cube_f16) {
    // float cubes of whole-warp fine DMs: the TMA-staged form
    bool done = false;
    int rc = DSB_OK;
#define DSB_DET_TMA(L)                                                                      \
  rc = det_tma_launch<L>((const float*)cube, n, n_f, npix, f_stride, t_stride, mask,         \
                         mask_f_stride, sig_f, sigma_inv, t_base, n_out, threshold, c, cap,  \
                         pix_off, count, l2, stream, &done)
    switch (log_maxw) {
      case 0: DSB_DET_TMA(0); break;
      case 1: DSB_DET_TMA(1); break;
      case 2: DSB_DET_TMA(2); break;
      case 3: DSB_DET_TMA(3); break;
      case 4: DSB_DET_TMA(4); break;
      case 5: DSB_DET_TMA(5); break;
      case 6: DSB_DET_TMA(6); break;
    }
#undef DSB_DET_TMA
    if (done || rc != DSB_OK) return rc;
  }
#define DSB_DET(L)                                                                        \
  do {                                                                                    \
    if (cube_f16)                                                                         \
      detect_kernel<L, __half><<<grid, 256, 0, stream>>>(                                 \
          (const __half*)cube, n, npix, inner, f_stride, t_stride, mask, mask_f_stride,   \
          sig_f, sigma_inv, t_base,                                                       \
          n_out, threshold, c, cap, pix_off, count, l2);                                   \
    else                                                                                  \
      detect_kernel<L, float><<<grid, 256, 0, stream>>>(                                  \
          (const float*)cube, n, npix, inner, f_stride, t_stride, mask, mask_f_stride,    \
          sig_f, sigma_inv, t_base,                                                       \
          n_out, threshold, c, cap, pix_off, count, l2);                                   \
  } while (0)
  switch (log_maxw) {
    case 0: DSB_DET(0); break;
    case 1: DSB_DET(1); break;
    case 2: DSB_DET(2); break;
    case 3: DSB_DET(3); break;
    case 4: DSB_DET(4); break;
    case 5: DSB_DET(5); break;
    case 6: DSB_DET(6); break;
  }
#undef DSB_DET
  return launch_status();
}

int dsb_clipped_std(const float* samples, int rows, int m, float n_sigma, int n_iter, float* out,
                    cudaStream_t stream) {
  if (!samples || !out || rows <= 0 || m <= 0 || n_iter < 0) return DSB_E_ARG;
  if (m > L1_MAX) return DSB_E_CAPACITY;
  L1Src src{samples, 0, 0, nullptr, nullptr, 1, 0};
  clipped_std_kernel<false><<<rows, L1_THREADS, 0, stream>>>(src, m, n_sigma, n_iter, out);
  return launch_status();
}

int dsb_layer1_sigma(const float* img, long long f_stride, long long t_stride, int n_f,
                     const int* times, int n_times, const int* pix, int n_pix, float n_sigma,
                     int n_iter, float* sigma, cudaStream_t stream) {
  if (!img || !times || !pix || !sigma || n_f <= 0 || n_times <= 0 || n_pix <= 0 || n_iter < 0)
    return DSB_E_ARG;
  if ((long long)n_times * n_pix > L1_MAX) return DSB_E_CAPACITY;
  L1Src src{img, f_stride, t_stride, times, pix, n_pix, 1};
  clipped_std_kernel<true><<<n_f, L1_THREADS, 0, stream>>>(src, n_times * n_pix, n_sigma, n_iter,
                                                            sigma);
  return launch_status();
}

}  // extern "C"

// ===========================================================================
// Boxcar S/N argmax without allocation.
//
// dsb_padded_cumsum + dsb_multi_boxcar_argmax need a caller-owned prefix-sum
// buffer of (n + max_w) x inner floats.  Some callers cannot allocate one: a
// host program that hands all of the GPU's memory to its own fixed arena at
// start-up, or a real-time loop where an allocation or free would stall
// every stream on the device (cudaFree synchronises the device).  For them,
// dsb_boxcar_argmax_noalloc keeps the prefix sums in the file-scope array
// below, DSB_NOALLOC_SCRATCH_BYTES (16 MiB) long, which every GPU that
// loads this file's device code holds until the process exits.
// ===========================================================================
#include <cuda.h>

#include <mutex>

static __device__ __align__(256) float g_boxcar_cs_scratch[DSB_NOALLOC_SCRATCH_BYTES / 4];

namespace {

// The scratch array's device address belongs to one CUDA context: after a
// cudaDeviceReset, or under another context on the same device, it is a
// different address.  So the cache is keyed on the current context's unique
// ID (cuCtxGetId, never reused within a process), looked up through the
// runtime's driver entry points so that the library needs no libcuda link.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

constexpr int kNoallocCache = 64;
struct NoallocEntry {
  unsigned long long ctx_id;
  float* ptr;
};
NoallocEntry g_noalloc_cache[kNoallocCache];
int g_noalloc_n = 0;
std::mutex g_noalloc_mu;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

bool load_ctx_fns() {
  if (g_ctx_get_current && g_ctx_get_id) return true;
  void* f1 = nullptr;
  void* f2 = nullptr;
  cudaDriverEntryPointQueryResult q1{}, q2{};
  if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
      cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
      q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
    cudaGetLastError();
    return false;
  }
  g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
  g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
  return true;
}

// The unique ID of the context current on this thread; 0 when there is none.
unsigned long long current_ctx_id() {
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array in the current context (the current
// device's primary context for a runtime caller), looked up on the first
// call in that context and cached.  Null on failure.
float* boxcar_cs_scratch() {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!load_ctx_fns()) return nullptr;
  unsigned long long id = current_ctx_id();
  if (id) {
    for (int i = 0; i < g_noalloc_n; ++i)
      if (g_noalloc_cache[i].ctx_id == id) return g_noalloc_cache[i].ptr;
  }
  // not seen yet (the runtime makes the device's context current here if
  // no context was)
  void* addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_boxcar_cs_scratch) != cudaSuccess || !addr) {
    cudaGetLastError();
    return nullptr;
  }
  if (!id) id = current_ctx_id();
  if (id) {
    // the oldest entry goes when the table is full (a process that made
    // more than 64 contexts); its context looks the address up again
    if (g_noalloc_n == kNoallocCache) {
      for (int i = 1; i < kNoallocCache; ++i) g_noalloc_cache[i - 1] = g_noalloc_cache[i];
      --g_noalloc_n;
    }
    g_noalloc_cache[g_noalloc_n++] = NoallocEntry{id, static_cast<float*>(addr)};
  }
  return static_cast<float*>(addr);
}

}  // namespace

extern "C" int dsb_boxcar_argmax_noalloc(const void* x, int x_f16, int n, long long inner,
                                         int max_w, const int* widths, const int* offsets,
                                         const float* sigma_inv, int K, int n_out, int t_base,
                                         void* out_max, int out_f16, void* out_win,
                                         cudaStream_t stream) {
  if (!x || !widths || !offsets || !sigma_inv || !out_max || !out_win) return DSB_E_ARG;
  if (n <= 0 || inner <= 0 || max_w < 1 || max_w > n || K < 1 || n_out <= 0 || t_base < 0 ||
      (long long)t_base + n_out > n)
    return DSB_E_ARG;
  // (n + max_w) rows of inner floats must fit the array; the sum is formed
  // in 64 bits and inner is bounded first, so neither the sum nor the
  // product can overflow
  constexpr long long kCap = (long long)(DSB_NOALLOC_SCRATCH_BYTES / 4);
  const long long rows = (long long)n + max_w;
  if (inner > kCap || rows * inner > kCap) return DSB_E_CAPACITY;
  float* cs = boxcar_cs_scratch();
  if (!cs) return DSB_E_CUDA;
  // padded_cumsum_kernel writes every one of the (n + max_w) x inner prefix
  // values, its zero padding rows included, so nothing left in the array by
  // an earlier call is read; the argmax below checks every row it reads
  // against those (n + max_w) rows.
  const int rc = dsb_padded_cumsum(x, x_f16, n, inner, max_w, cs, stream);
  if (rc != DSB_OK) return rc;
  const long long total = (long long)n_out * inner;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (out_f16)
    multi_boxcar_argmax_kernel<true, true><<<grid, 256, 0, stream>>>(
        cs, inner, widths, offsets, sigma_inv, K, n_out, t_base, out_max, (int16_t*)out_win,
        rows);
  else
    multi_boxcar_argmax_kernel<false, true><<<grid, 256, 0, stream>>>(
        cs, inner, widths, offsets, sigma_inv, K, n_out, t_base, out_max, (int16_t*)out_win,
        rows);
  return launch_status();
}
