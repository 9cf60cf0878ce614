// Gridding, stage-1 coarse-DM shift + grid, static-sky subtraction and the
// stage-2 per-coarse-DM delay (sm_100a).
//
// Drop-in forms (reference layouts):
//   dsb_grid_vis          FastVisGridder.compute       (n_fv, nbase, C) -> (n_fv, n_filled)
//   dsb_dedisp_vis        Stage1MultiDMCoarseDM window (T, nbase, C)    -> (n_dm, T_d, n_filled)
//   dsb_static_sky        StaticSkyMean.apply          (n_fv, n_filled) -> same
//   dsb_stage2_roll       Stage2InterChgroupShiftFifo  ring of cubes    -> aligned cube
// Pipeline form (time-major rows, ring buffers indexed by absolute time):
//   dsb_stage1_rows       per-subband gridded rows Y -> per-(chgroup, DM,
//                         cell) rows written at t + shift2 into the stage-2
//                         ring, static-sky subtraction fused.
#include "dsb_common.cuh"

#include <algorithm>

namespace {

__global__ void grid_vis_kernel(const float2* __restrict__ vis, int n_fv, long long nsrc,
                                const int* __restrict__ off, const int* __restrict__ src,
                                int n_filled, float2* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_fv * n_filled) return;
  const int f = (int)(idx / n_filled), cell = (int)(idx % n_filled);
  const float2* v = vis + (size_t)f * nsrc;
  float re = 0.f, im = 0.f;
  for (int j = off[cell]; j < off[cell + 1]; ++j) {
    const float2 x = v[src[j]];
    re += x.x;
    im += x.y;
  }
  out[idx] = make_float2(re, im);
}

// out[d, t, cell] = sum_{src in cell} vis_joined[t + shift[s(src), d], src]
// where vis_joined = concat(prev[0:n_prev], cur) along time.
__global__ void dedisp_vis_kernel(const float2* __restrict__ prev, const float2* __restrict__ cur,
                                  int n_prev, long long nsrc, int ceff,
                                  const int* __restrict__ off, const int* __restrict__ src,
                                  const int* __restrict__ shifts, int n_dm, int n_filled,
                                  int t_dedisp, float2* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_d = (long long)t_dedisp * n_filled;
  if (idx >= per_d * n_dm) return;
  const int d = (int)(idx / per_d);
  const long long r = idx % per_d;
  const int t = (int)(r / n_filled), cell = (int)(r % n_filled);
  float re = 0.f, im = 0.f;
  for (int j = off[cell]; j < off[cell + 1]; ++j) {
    const int sj = src[j];
    const int tt = t + shifts[(sj % ceff) * n_dm + d];
    const float2 x = tt < n_prev ? prev[(size_t)tt * nsrc + sj] : cur[(size_t)(tt - n_prev) * nsrc + sj];
    re += x.x;
    im += x.y;
  }
  out[idx] = make_float2(re, im);
}

// Static-sky mean (per cell): mean of the past `count` block means held in
// ring[cell*window + w] (float64), subtracted once `subtract` is set; this
// block's float64 time-mean is written to ring[cell*window + head].
__global__ void static_sky_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                  int n_t, int n_cells, double2* __restrict__ ring, int window,
                                  int head, int count, int subtract) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= n_cells) return;
  double2 m = make_double2(0.0, 0.0);
  if (subtract && count > 0) {
    for (int w = 0; w < count; ++w) {
      const double2 r = ring[(size_t)cell * window + w];
      m.x += r.x;
      m.y += r.y;
    }
    m.x /= count;
    m.y /= count;
  }
  double sr = 0.0, si = 0.0;
  for (int t = 0; t < n_t; ++t) {
    const float2 x = in[(size_t)t * n_cells + cell];
    sr += x.x;
    si += x.y;
    if (subtract && count > 0)
      out[(size_t)t * n_cells + cell] =
          make_float2((float)((double)x.x - m.x), (float)((double)x.y - m.y));
    else
      out[(size_t)t * n_cells + cell] = x;
  }
  ring[(size_t)cell * window + head] = make_double2(sr / n_t, si / n_t);
}

// Stage-2 aligned cube: out[c, t, :] = stream_c[t - shift[c]] where the
// stream is the concatenation of past cubes; hist[c][j] points at the cube
// pushed j ticks ago (j = 0 newest).  warm[c] == 0 -> zeros.
__global__ void stage2_roll_kernel(const float2* const* __restrict__ hist, int depth,
                                   const int* __restrict__ kblk, const int* __restrict__ rsmp,
                                   const int* __restrict__ warm, int n_dm, int t_len,
                                   long long inner, float2* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_c = (long long)t_len * inner;
  if (idx >= per_c * n_dm) return;
  const int c = (int)(idx / per_c);
  const long long r = idx % per_c;
  const int t = (int)(r / inner);
  const long long e = r % inner;
  float2 v = make_float2(0.f, 0.f);
  if (warm[c]) {
    const int k = kblk[c], rr = rsmp[c];
    int j, ts;
    if (t < rr) {
      j = k + 1;
      ts = t_len - rr + t;
    } else {
      j = k;
      ts = t - rr;
    }
    if (j < depth) {
      const float2* cube = hist[j];
      v = cube[((size_t)c * t_len + ts) * inner + e];
    }
  }
  out[idx] = v;
}

// Pipeline stage 1 over per-subband gridded rows, time-major rings:
//   Y[(t & y_mask) * y_rows + y_base[g] + s * pitch[g] + cell],
//   D[seg_base[g*n_dm + d] + (t mod seg_depth[g*n_dm + d]) * pitch[g] + cell]
// (each (chgroup, coarse DM) a ring segment as deep as its own stage-2 delay
// needs); the sky ring is indexed by d_base[g] + d * pitch[g] + cell.
// Rows are dense per (chgroup, subband) and (chgroup, coarse DM) with an
// even pitch, so one thread owns two adjacent cells (16-byte loads and
// stores) and the 32 lanes of a warp read 512 contiguous bytes.  Blocks
// never straddle chgroups; one grid row per coarse DM.  Time is walked in
// tiles of S1_TT samples: for each subband the tile's S1_TT loads are
// independent.
struct S1Args {
  const float2* Y;
  long long y_rows, y_mask;
  const int* blk_g;       // chgroup of each block
  const int* blk_c0;      // first cell of each block (even)
  const int* y_base;      // (G) first Y row of the chgroup (even)
  const int* pitch;       // (G) even row pitch between subbands / coarse DMs
  const int* shift1;      // (G, ceff, n_dm)
  const int* shift2;      // (G, n_dm)
  const int* d_base;      // (G) first sky-ring row of the chgroup (even)
  const int* n_filled;    // (G)
  float2* D;
  const long long* seg_base;  // (G * n_dm) first element of each ring segment (even)
  const int* seg_depth;       // (G * n_dm) time slots of each segment
  long long t0;           // absolute time of the first output
  int n_t, n_dm, ceff;
  double2* sky_ring;      // (D rows, window) or null
  int sky_window, sky_head, sky_count, sky_subtract;
};

constexpr int S1_THREADS = 128;
constexpr int S1_MAX_C = 64;
constexpr int S1_TT = 8;

__global__ void __launch_bounds__(S1_THREADS) stage1_rows_kernel(const S1Args A) {
  __shared__ int s_sh[S1_MAX_C];
  const int g = A.blk_g[blockIdx.x];
  const int d = blockIdx.y;
  const int nf = A.n_filled[g];
  const int pitch = A.pitch[g];
  const int cl = A.blk_c0[blockIdx.x] + 2 * threadIdx.x;
  const int ceff = A.ceff;
  for (int s = threadIdx.x; s < ceff; s += S1_THREADS)
    s_sh[s] = A.shift1[(g * ceff + s) * A.n_dm + d];
  __syncthreads();
  if (cl >= nf) return;  // cl + 1 <= pitch - 1: a pad cell at most
  const float4* Y4 = reinterpret_cast<const float4*>(A.Y);
  float4* D4 = reinterpret_cast<float4*>(A.D);
  const long long y_rows2 = A.y_rows / 2;
  const long long seg = (long long)A.seg_base[g * A.n_dm + d] + cl;
  const long long dep = A.seg_depth[g * A.n_dm + d];
  const long long ycol2 = (A.y_base[g] + cl) / 2;
  const long long drow = (long long)A.d_base[g] + (long long)d * pitch + cl;
  double mr[2] = {0.0, 0.0}, mi[2] = {0.0, 0.0};
  const bool sub = A.sky_ring && A.sky_subtract && A.sky_count > 0;
  if (sub) {
    for (int c = 0; c < 2; ++c) {
      for (int w = 0; w < A.sky_count; ++w) {
        const double2 r = A.sky_ring[(drow + c) * A.sky_window + w];
        mr[c] += r.x;
        mi[c] += r.y;
      }
      mr[c] /= A.sky_count;
      mi[c] /= A.sky_count;
    }
  }
  const int sh2 = A.shift2[g * A.n_dm + d];
  double sr[2] = {0.0, 0.0}, si[2] = {0.0, 0.0};
  for (int t = 0; t < A.n_t; t += S1_TT) {
    const long long ta = A.t0 + t;
    long long wpos = (ta + sh2) % dep;  // write slot of time ta (wraps below)
    if (wpos < 0) wpos += dep;
    float4 acc[S1_TT];
#pragma unroll
    for (int i = 0; i < S1_TT; ++i) acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int s = 0; s < ceff; ++s) {
      const long long col = ycol2 + (long long)s * (pitch / 2);
      const long long p0 = ta + s_sh[s];
#pragma unroll
      for (int i = 0; i < S1_TT; ++i) {
        const float4 v = Y4[((p0 + i) & A.y_mask) * y_rows2 + col];
        acc[i].x += v.x;
        acc[i].y += v.y;
        acc[i].z += v.z;
        acc[i].w += v.w;
      }
    }
#pragma unroll
    for (int i = 0; i < S1_TT; ++i) {
      if (t + i < A.n_t) {
        const float4 a = acc[i];
        sr[0] += a.x;
        si[0] += a.y;
        sr[1] += a.z;
        si[1] += a.w;
        float4 o = a;
        if (sub)
          o = make_float4((float)((double)a.x - mr[0]), (float)((double)a.y - mi[0]),
                          (float)((double)a.z - mr[1]), (float)((double)a.w - mi[1]));
        long long slot = wpos + i;
        if (slot >= dep) slot -= dep;
        D4[(seg + slot * pitch) / 2] = o;
      }
    }
  }
  if (A.sky_ring) {
    A.sky_ring[drow * A.sky_window + A.sky_head] = make_double2(sr[0] / A.n_t, si[0] / A.n_t);
    A.sky_ring[(drow + 1) * A.sky_window + A.sky_head] =
        make_double2(sr[1] / A.n_t, si[1] / A.n_t);
  }
}

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

}  // namespace

extern "C" {

int dsb_grid_vis(const void* vis, int n_fv, long long nsrc, const int* cell_off,
                 const int* cell_src, int n_filled, void* out, cudaStream_t stream) {
  if (!vis || !out || !cell_off || !cell_src || n_fv <= 0 || n_filled < 0) return DSB_E_ARG;
  const long long n = (long long)n_fv * n_filled;
  if (n == 0) return DSB_OK;
  grid_vis_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      (const float2*)vis, n_fv, nsrc, cell_off, cell_src, n_filled, (float2*)out);
  return launch_status();
}

int dsb_dedisp_vis(const void* prev, const void* cur, int n_prev, long long nsrc, int ceff,
                   const int* cell_off, const int* cell_src, const int* shifts, int n_dm,
                   int n_filled, int t_dedisp, void* out, cudaStream_t stream) {
  if (!cur || !out || !cell_off || !cell_src || !shifts || ceff <= 0 || n_dm <= 0) return DSB_E_ARG;
  if (n_prev > 0 && !prev) return DSB_E_ARG;
  const long long n = (long long)n_dm * t_dedisp * n_filled;
  if (n <= 0) return DSB_OK;
  dedisp_vis_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      (const float2*)prev, (const float2*)cur, n_prev, nsrc, ceff, cell_off, cell_src, shifts,
      n_dm, n_filled, t_dedisp, (float2*)out);
  return launch_status();
}

int dsb_static_sky(const void* in, void* out, int n_t, int n_cells, void* ring, int window,
                   int head, int count, int subtract, cudaStream_t stream) {
  if (!in || !out || !ring || n_t <= 0 || n_cells < 0 || window <= 0) return DSB_E_ARG;
  if (head < 0 || head >= window || count < 0 || count > window) return DSB_E_ARG;
  if (n_cells == 0) return DSB_OK;
  static_sky_kernel<<<(n_cells + 127) / 128, 128, 0, stream>>>(
      (const float2*)in, (float2*)out, n_t, n_cells, (double2*)ring, window, head, count,
      subtract);
  return launch_status();
}

int dsb_stage2_roll(const void* const* hist, int depth, const int* kblk, const int* rsmp,
                    const int* warm, int n_dm, int t_len, long long inner, void* out,
                    cudaStream_t stream) {
  if (!hist || !kblk || !rsmp || !warm || !out || depth <= 0 || n_dm <= 0 || t_len <= 0)
    return DSB_E_ARG;
  const long long n = (long long)n_dm * t_len * inner;
  if (n == 0) return DSB_OK;
  stage2_roll_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      (const float2* const*)hist, depth, kblk, rsmp, warm, n_dm, t_len, inner, (float2*)out);
  return launch_status();
}

int dsb_stage1_rows(const void* Y, long long y_rows, long long y_mask, int n_blocks,
                    const int* blk_g, const int* blk_c0, const int* y_base, const int* pitch,
                    const int* shift1, const int* shift2, const int* d_base, const int* n_filled,
                    void* D, const long long* seg_base, const int* seg_depth, long long t0,
                    int n_t, int n_dm,
                    int ceff, void* sky_ring, int sky_window, int sky_head, int sky_count,
                    int sky_subtract, cudaStream_t stream) {
  if (!Y || !D || !blk_g || !blk_c0 || !y_base || !pitch || !shift1 || !shift2 ||
      !d_base || !n_filled || !seg_base || !seg_depth || n_t <= 0 || n_dm <= 0 || ceff <= 0)
    return DSB_E_ARG;
  // two cells per 16-byte access: rings 16-byte aligned, row counts even
  if ((reinterpret_cast<uintptr_t>(Y) & 15) || (reinterpret_cast<uintptr_t>(D) & 15) ||
      (y_rows & 1))
    return DSB_E_ARG;
  if (ceff > S1_MAX_C) return DSB_E_CAPACITY;
  if (sky_ring && (sky_window <= 0 || sky_head < 0 || sky_head >= sky_window ||
                   sky_count < 0 || sky_count > sky_window))
    return DSB_E_ARG;
  if (n_blocks <= 0) return DSB_OK;
  S1Args A{};
  A.Y = (const float2*)Y; A.y_rows = y_rows; A.y_mask = y_mask;
  A.blk_g = blk_g; A.blk_c0 = blk_c0; A.y_base = y_base; A.pitch = pitch;
  A.shift1 = shift1; A.shift2 = shift2; A.d_base = d_base; A.n_filled = n_filled;
  A.D = (float2*)D; A.seg_base = seg_base; A.seg_depth = seg_depth;
  A.t0 = t0; A.n_t = n_t; A.n_dm = n_dm; A.ceff = ceff;
  A.sky_ring = (double2*)sky_ring; A.sky_window = sky_window; A.sky_head = sky_head;
  A.sky_count = sky_count; A.sky_subtract = sky_subtract;
  dim3 grid(n_blocks, n_dm);
  stage1_rows_kernel<<<grid, S1_THREADS, 0, stream>>>(A);
  return launch_status();
}

int dsb_stage1_block_size(void) { return 2 * S1_THREADS; }

}  // extern "C"
