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
#include <type_traits>

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
//
// A CTA owns 4 adjacent cells of one chgroup and a group of DG coarse
// DMs, and walks the output times in tiles of S1_TT.  For each tile it
// stages every subband's Y samples that any of its DMs needs (the tile plus
// the spread of that subband's shifts over the DM group) in shared memory,
// two planes of two cells, and then every (DM, time) output of the tile sums
// its ceff subbands from there: each Y sample is read from L2 once per DM
// group instead of once per DM.  Thread (dl, ln) = (tid / L, tid % L), with
// L = 256 / DG lanes per DM, owns DM dl of the group and times ln, ln + L,
// ...; DG is 32, 16 or 8: the largest whose windows fit in shared memory
// (a wide DM spread per group, as with few coarse DMs over a wide range,
// needs a smaller group); its D writes are whole
// 32-byte sectors (4 cells).
struct S1Args {
  const float2* Y;
  long long y_rows, y_mask;
  const int* blk_g;       // chgroup of each block
  const int* blk_c0;      // first cell of each block (a multiple of 4)
  const int* y_base;      // (G) first Y row of the chgroup (a multiple of 4)
  const int* pitch;       // (G) row pitch between subbands / coarse DMs (a multiple of 4)
  const int* shift1;      // (G, ceff, n_dm)
  const int* shift2;      // (G, n_dm)
  const int* d_base;      // (G) first sky-ring row of the chgroup
  const int* n_filled;    // (G)
  void* D;                // complex64 elements, or (BF16) bf16 re/im pairs in 32 bits
  const long long* seg_base;  // (G * n_dm) first element of each ring segment (a multiple of 4)
  const int* seg_depth;       // (G * n_dm) time slots of each segment
  float* amax;            // (G * n_dm) or null: raised to the largest |part| written
  long long t0;           // absolute time of the first output
  int n_t, n_dm, ceff;
  int win_len;            // S1_TT + largest shift spread over a DM group
  double2* sky_ring;      // (D rows, window) or null
  int sky_window, sky_head, sky_count, sky_subtract;
  int* status;
};

constexpr int S1_THREADS = 256;
constexpr int S1_MAX_C = 64;
constexpr int S1_TT = 64;   // output times per tile
constexpr int S1_DG = 32;   // largest DM group (coarse DMs per CTA)

__host__ __device__ inline size_t s1_smem_bytes(int ceff, int dg, int win_len) {
  return (size_t)ceff * dg * 4 + (size_t)S1_MAX_C * 8 + (size_t)ceff * win_len * 32 + 16;
}

template <bool BF16, int DG>
__global__ void __launch_bounds__(S1_THREADS) stage1_rows_kernel(const S1Args A) {
  constexpr int L = S1_THREADS / DG;  // time lanes per DM
  static_assert(L >= 8 && L <= 32 && S1_TT % L == 0, "unsupported DM group");
  extern __shared__ __align__(16) uint8_t s1_smem[];
  const int ceff = A.ceff;
  int* s_sh = reinterpret_cast<int*>(s1_smem);              // [s][dl] shift - lo[s]
  int* s_lo = s_sh + ceff * DG;                             // [s] smallest shift
  int* s_len = s_lo + S1_MAX_C;                             // [s] window length
  float4* win0 = reinterpret_cast<float4*>(s1_smem + ((size_t)ceff * DG * 4 +
                                                      (size_t)S1_MAX_C * 8 + 15) / 16 * 16);
  float4* win1 = win0 + (size_t)ceff * A.win_len;            // cells 2-3

  const int g = A.blk_g[blockIdx.x];
  const int c0 = A.blk_c0[blockIdx.x];
  const int dg0 = blockIdx.y * DG;
  const int nd = min(DG, A.n_dm - dg0);
  const int pitch = A.pitch[g];
  const int tid = threadIdx.x;
  for (int sb = tid; sb < ceff; sb += S1_THREADS) {
    const int* sh = A.shift1 + ((long long)g * ceff + sb) * A.n_dm + dg0;
    int lo = sh[0], hi = sh[0];
    for (int dl = 1; dl < nd; ++dl) {
      lo = min(lo, sh[dl]);
      hi = max(hi, sh[dl]);
    }
    s_lo[sb] = lo;
    s_len[sb] = S1_TT + hi - lo;
  }
  __syncthreads();
  // a window longer than the caller sized the shared memory for: flag, stop
  bool fits = true;
  for (int sb = 0; sb < ceff; ++sb) fits = fits && s_len[sb] <= A.win_len;
  if (!fits) {
    if (tid == 0) dsb_flag(A.status, DSB_E_CAPACITY);
    return;
  }
  for (int i = tid; i < ceff * DG; i += S1_THREADS) {
    const int sb = i / DG, dl = i % DG;
    s_sh[i] = dl < nd ? A.shift1[((long long)g * ceff + sb) * A.n_dm + dg0 + dl] - s_lo[sb] : 0;
  }

  const int dl = tid / L, ln = tid % L;
  const bool active = dl < nd;
  const int d = dg0 + (active ? dl : 0);
  const int gd = g * A.n_dm + d;
  const long long seg = A.seg_base[gd] + c0;
  const long long dep = A.seg_depth[gd];
  const int sh2 = A.shift2[gd];
  const long long drow = (long long)A.d_base[g] + (long long)d * pitch + c0;
  double mr[4] = {0, 0, 0, 0}, mi[4] = {0, 0, 0, 0};
  const bool sub = A.sky_ring && A.sky_subtract && A.sky_count > 0;
  if (sub && active) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      for (int w = 0; w < A.sky_count; ++w) {
        const double2 r = A.sky_ring[(drow + c) * A.sky_window + w];
        mr[c] += r.x;
        mi[c] += r.y;
      }
      mr[c] /= A.sky_count;
      mi[c] /= A.sky_count;
    }
  }
  double sr[4] = {0, 0, 0, 0}, si[4] = {0, 0, 0, 0};
  float amax = 0.f;  // largest |part| this thread writes
  const float4* Y4 = reinterpret_cast<const float4*>(A.Y);
  const long long ycol = (long long)A.y_base[g] + c0;   // a multiple of 4

  for (int tt = 0; tt < A.n_t; tt += S1_TT) {
    __syncthreads();  // the previous tile's windows are no longer read
    // stage the windows: entry (sb, tau) = Y at time t0 + tt + lo[sb] + tau,
    // flattened over (sb, tau) so that each thread's loads are independent
    {
      constexpr int U = 4;
      const int n_e = ceff * A.win_len;
      for (int e0 = 0; e0 < n_e; e0 += U * S1_THREADS) {
        float4 v0[U], v1[U];
        int ei[U];
#pragma unroll
        for (int q = 0; q < U; ++q) {
          const int e = e0 + q * S1_THREADS + tid;
          ei[q] = -1;
          if (e < n_e) {
            const int sb = e / A.win_len, tau = e - sb * A.win_len;
            if (tau < s_len[sb]) {
              const long long r2 = ((((A.t0 + tt + s_lo[sb] + tau) & A.y_mask) * A.y_rows) +
                                    ycol + (long long)sb * pitch) / 2;
              if (DSB_INB(r2 + 1, (A.y_mask + 1) * A.y_rows / 2, A.status)) {
                v0[q] = Y4[r2];
                v1[q] = Y4[r2 + 1];
                ei[q] = e;
              }
            }
          }
        }
#pragma unroll
        for (int q = 0; q < U; ++q) {
          if (ei[q] >= 0) {
            win0[ei[q]] = v0[q];
            win1[ei[q]] = v1[q];
          }
        }
      }
    }
    __syncthreads();
    if (!active) continue;
    long long slot = (A.t0 + tt + ln + sh2) % dep;
    if (slot < 0) slot += dep;
    for (int k = 0; k < S1_TT / L; ++k, slot += L) {
      if (slot >= dep) slot -= dep;
      const int tl = ln + L * k;
      if (tt + tl >= A.n_t) break;
      float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
      for (int sb = 0; sb < ceff; ++sb) {
        const int idx = sb * A.win_len + tl + s_sh[sb * DG + dl];
        const float4 v0 = win0[idx], v1 = win1[idx];
        a0 = f4_add(a0, v0);  // packed pairs: 4 adds instead of 8
        a1 = f4_add(a1, v1);
      }
      sr[0] += a0.x; si[0] += a0.y; sr[1] += a0.z; si[1] += a0.w;
      sr[2] += a1.x; si[2] += a1.y; sr[3] += a1.z; si[3] += a1.w;
      float4 o0 = a0, o1 = a1;
      if (sub) {
        o0 = make_float4((float)((double)a0.x - mr[0]), (float)((double)a0.y - mi[0]),
                         (float)((double)a0.z - mr[1]), (float)((double)a0.w - mi[1]));
        o1 = make_float4((float)((double)a1.x - mr[2]), (float)((double)a1.y - mi[2]),
                         (float)((double)a1.z - mr[3]), (float)((double)a1.w - mi[3]));
      }
      amax = fmaxf(amax, fmaxf(fmaxf(fabsf(o0.x), fabsf(o0.y)), fmaxf(fabsf(o0.z), fabsf(o0.w))));
      amax = fmaxf(amax, fmaxf(fmaxf(fabsf(o1.x), fabsf(o1.y)), fmaxf(fabsf(o1.z), fabsf(o1.w))));
      const long long o = seg + slot * pitch;  // element of cell c0, a multiple of 4
      if (!(DSB_INB(slot, dep, A.status) && DSB_INB(c0 + 3, pitch, A.status))) continue;
      if constexpr (BF16) {
        reinterpret_cast<uint4*>(A.D)[o / 4] =
            make_uint4(bf16_pair(o0.x, o0.y), bf16_pair(o0.z, o0.w), bf16_pair(o1.x, o1.y),
                       bf16_pair(o1.z, o1.w));
      } else {
        float4* D4 = reinterpret_cast<float4*>(A.D);
        D4[o / 2] = o0;
        D4[o / 2 + 1] = o1;
      }
    }
  }
  // the bound of the (chgroup, DM) rows: max over the L lanes that share
  // the DM, one atomic per DM and block (non-negative floats order as ints)
  if (A.amax) {
#pragma unroll
    for (int o = 1; o < L; o <<= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if (active && ln == 0) atomicMax(reinterpret_cast<int*>(A.amax) + gd, __float_as_int(amax));
  }
  // sky: block mean of every (DM, cell) over the chunk, summed over the L
  // lanes that share the DM (L-aligned inside the warp)
  if (A.sky_ring) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
#pragma unroll
      for (int o = 1; o < L; o <<= 1) {
        sr[c] += __shfl_xor_sync(0xffffffffu, sr[c], o);
        si[c] += __shfl_xor_sync(0xffffffffu, si[c], o);
      }
    }
    if (active && ln == 0) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        A.sky_ring[(drow + c) * A.sky_window + A.sky_head] =
            make_double2(sr[c] / A.n_t, si[c] / A.n_t);
    }
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
                    void* D, int d_bf16, const long long* seg_base, const int* seg_depth,
                    float* amax, long long t0, int n_t, int n_dm, int ceff, int dm_group, int max_spread,
                    void* sky_ring, int sky_window,
                    int sky_head, int sky_count, int sky_subtract, int* status,
                    cudaStream_t stream) {
  if (!Y || !D || !blk_g || !blk_c0 || !y_base || !pitch || !shift1 || !shift2 ||
      !d_base || !n_filled || !seg_base || !seg_depth || n_t <= 0 || n_dm <= 0 || ceff <= 0 ||
      max_spread < 0 || (dm_group != 32 && dm_group != 16 && dm_group != 8))
    return DSB_E_ARG;
  // four cells per 32-byte access: rings 16-byte aligned, row counts multiples of 4
  if ((reinterpret_cast<uintptr_t>(Y) & 15) || (reinterpret_cast<uintptr_t>(D) & 15) ||
      (y_rows & 3))
    return DSB_E_ARG;
  if (ceff > S1_MAX_C) return DSB_E_CAPACITY;
  const int win_len = S1_TT + max_spread;
  const size_t smem = s1_smem_bytes(ceff, dm_group, win_len);
  if (smem > 227 * 1024) return DSB_E_CAPACITY;
  if (sky_ring && (sky_window <= 0 || sky_head < 0 || sky_head >= sky_window ||
                   sky_count < 0 || sky_count > sky_window))
    return DSB_E_ARG;
  if (n_blocks <= 0) return DSB_OK;
  S1Args A{};
  A.Y = (const float2*)Y; A.y_rows = y_rows; A.y_mask = y_mask;
  A.blk_g = blk_g; A.blk_c0 = blk_c0; A.y_base = y_base; A.pitch = pitch;
  A.shift1 = shift1; A.shift2 = shift2; A.d_base = d_base; A.n_filled = n_filled;
  A.D = D; A.seg_base = seg_base; A.seg_depth = seg_depth; A.amax = amax;
  A.t0 = t0; A.n_t = n_t; A.n_dm = n_dm; A.ceff = ceff; A.win_len = win_len;
  A.sky_ring = (double2*)sky_ring; A.sky_window = sky_window; A.sky_head = sky_head;
  A.sky_count = sky_count; A.sky_subtract = sky_subtract; A.status = status;
  auto pick = [&](auto bf) {
    constexpr bool B = decltype(bf)::value;
    return dm_group == 32 ? stage1_rows_kernel<B, 32>
         : dm_group == 16 ? stage1_rows_kernel<B, 16> : stage1_rows_kernel<B, 8>;
  };
  auto kern = d_bf16 ? pick(std::true_type{}) : pick(std::false_type{});
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return DSB_E_CUDA;
  dim3 grid(n_blocks, (n_dm + dm_group - 1) / dm_group);
  kern<<<grid, S1_THREADS, smem, stream>>>(A);
  return launch_status();
}

int dsb_stage1_block_size(void) { return 4; }
int dsb_stage1_dm_group(void) { return S1_DG; }

long long dsb_stage1_smem_bytes(int ceff, int dm_group, int max_spread) {
  if (ceff <= 0 || ceff > S1_MAX_C || max_spread < 0 ||
      (dm_group != 32 && dm_group != 16 && dm_group != 8))
    return -1;
  return (long long)s1_smem_bytes(ceff, dm_group, S1_TT + max_spread);
}

}  // extern "C"
