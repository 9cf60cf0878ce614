// 4-bit unpack and X-engine correlator kernels (sm_100a).
//
//  * dsb_unpack_int4   : on-wire (npkt, nant, nchan, 2t, 2p) int4 pairs ->
//                        GEMM layout (nchan, 2t, 2p, npkt, nant) int8/fp16/fp32.
//  * dsb_corr_split    : correlator on GEMM-layout voltages (any of the three
//                        dtypes), Stokes-I + channel sum or 2-pol output.
//  * dsb_corr_tc       : fused unpack + correlate from raw on-wire bytes on the
//                        5th-generation tensor cores (tcgen05.mma kind::i8,
//                        int32 accumulators in tensor memory), Stokes-I and
//                        channel sum folded into the contraction dimension.
//                        Epilogue writes strided complex64 visibilities, or
//                        grids them per subband into time-major rows.
#include "dsb_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <type_traits>

namespace {

// ===========================================================================
// unpack
// ===========================================================================
template <typename T>
DSB_DEV T from_code(int v, float scale);
template <>
DSB_DEV int8_t from_code<int8_t>(int v, float) { return (int8_t)v; }
template <>
DSB_DEV __half from_code<__half>(int v, float scale) {
  return __float2half_rn((float)v * scale);
}
template <>
DSB_DEV float from_code<float>(int v, float scale) { return (float)v * scale; }

// Tile: 32 (pkt*nant) rows x 32 channels; smem transpose so that the
// 4-byte raw words are read along channels and the outputs are written
// along (pkt, ant).
template <typename T>
__global__ void unpack_kernel(const uint32_t* __restrict__ raw, int rows, int nchan, float scale,
                              T* __restrict__ ore, T* __restrict__ oim) {
  __shared__ uint32_t tile[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int i = ty; i < 32; i += 8) {
    int r = r0 + i, c = c0 + tx;
    tile[i][tx] = (r < rows && c < nchan) ? raw[(size_t)r * nchan + c] : 0u;
  }
  __syncthreads();
  const size_t plane = (size_t)rows;  // elements per (c, t, pol) plane
  for (int i = ty; i < 32; i += 8) {
    int c = c0 + i, r = r0 + tx;
    if (c >= nchan || r >= rows) continue;
    uint32_t w = tile[tx][i];
#pragma unroll
    for (int tp = 0; tp < 4; ++tp) {  // byte tp = (t, pol)
      int b = (w >> (8 * tp)) & 0xFF;
      int re = (b & 8) ? (b & 0xF) - 16 : (b & 0xF);
      int hi = b >> 4;
      int im = (hi & 8) ? hi - 16 : hi;
      size_t o = ((size_t)c * 4 + tp) * plane + r;
      ore[o] = from_code<T>(re, scale);
      oim[o] = from_code<T>(im, scale);
    }
  }
}

// ===========================================================================
// tensor-core correlator (tcgen05, kind::i8)
// ===========================================================================
constexpr int TC_THREADS = 256;
constexpr int TC_TMEM_COLS = 512;   // two accumulators of <= 256 columns
constexpr int TC_SMEM_BUDGET = 224 * 1024;
constexpr int TC_PRE = 4;          // 16-byte raw loads per thread per item (nant <= 128)
constexpr int TC_CAP_ROWS = 4096;  // gridding rows of one (chgroup, subband) kept in smem
// Every CTA requests more than half an SM's shared memory so that exactly
// one CTA (and one 512-column tensor-memory allocation) lives on each SM.
constexpr int TC_MIN_SMEM = 120 * 1024;

struct TcArgs {
  const uint8_t* raw;
  long long raw_g_stride;  // bytes
  int n_chgroup, npkt, nant, nchan, t_int, csf;
  int ceff, ppfv, n_fv, rows, kc, n_chunks, nkblk, stage_bytes, nstage, n_mma;
  int unit_order;  // 0: fast-vis tile fastest, 1: summed channel fastest
  // mode 0
  float2* out;
  long long o_g, o_f, o_b, o_s;
  // mode 1
  const int* yoff;    // (n_chgroup*ceff) first global row of the group
  const int* ycnt;    // (n_chgroup*ceff) rows in the group
  const int* row_off; // (n_rows + 1) CSR over rows: baselines gridded into each row
  const int* row_bls; // baseline index of each CSR entry
  float2* yout;
  long long y_t_stride;
  long long t_base;
  long long t_mask;
  // (n_chgroup, ceff, nant) complex gains or null: every visibility is
  // multiplied by g_a conj(g_b) of its subband before it is gridded
  const float2* gains;
  // raw staging by TMA (tma != 0): each item's raw bytes, ppk packets x nant
  // antennas x csf channels x 4 bytes, arrive by one 4-D tensor copy into one
  // of nraw shared-memory stages of raw_stage bytes, nraw - 1 items ahead
  int tma, ppk, raw_stage, nraw;
  int* status;
};

DSB_DEV void tc_unit_coords(const TcArgs& A, int u, int& g, int& f, int& s) {
  const int per_g = A.n_fv * A.ceff;
  g = u / per_g;
  const int r = u % per_g;
  if (A.unit_order == 0) {
    f = r % A.n_fv;
    s = r / A.n_fv;
  } else {
    s = r % A.ceff;
    f = r / A.ceff;
  }
}

// The 16-byte raw words of one K chunk of one unit (vectorised path: csf and
// nchan multiples of 4): thread t loads words t, t + 256, ... of the chunk.
DSB_DEV void tc_load(const TcArgs& A, int g, int f, int s, int q, uint4 (&w)[TC_PRE]) {
  const int nv = A.kc / 16;
  const uint8_t* base = A.raw + (size_t)g * A.raw_g_stride;
#pragma unroll
  for (int r = 0; r < TC_PRE; ++r) {
    const int idx = threadIdx.x + r * TC_THREADS;
    if (idx < A.nant * nv) {
      const int a = idx / nv, v = idx % nv;
      const int j = q * (A.kc / 4) + v * 4;
      const int p = j / A.csf, c = j % A.csf;
      w[r] = __ldg(reinterpret_cast<const uint4*>(
          base + ((((size_t)(f * A.ppfv + p) * A.nant + a) * A.nchan + (size_t)s * A.csf + c) * 4)));
    }
  }
}

// Per-thread offsets of the vectorised fill, computed once per kernel (no
// divisions per item): byte offset of word r of chunk 0 inside a unit's raw
// data, and the four shared-memory destinations of its unpacked words.  Valid
// when a chunk covers whole packets (kc/4 a multiple of csf): chunk q is then
// chunk 0 moved by q * (kc/4/csf) packets.
struct TcFillPlan {
  int ld[TC_PRE];
  int lds[TC_PRE];    // the same word in a TMA raw stage [ppk][nant][csf * 4 bytes]
  uint32_t st[TC_PRE][4];
  long long q_step;   // bytes between chunks
  long long f_step;   // bytes between fast-vis tiles
  int s_step;         // bytes between summed channels
};

DSB_DEV void tc_fill_plan(const TcArgs& A, TcFillPlan& P) {
  const int nv = A.kc / 16;
  const uint32_t region = (uint32_t)A.rows * 128u;
  const long long pkt = (long long)A.nant * A.nchan * 4;
#pragma unroll
  for (int r = 0; r < TC_PRE; ++r) {
    const int idx = threadIdx.x + r * TC_THREADS;
    const int a = idx / nv, v = idx % nv;
    const int p = (v * 4) / A.csf, c = (v * 4) % A.csf;
    P.ld[r] = (int)(((long long)p * A.nant + a) * A.nchan * 4 + (long long)c * 4);
    P.lds[r] = ((p * A.nant + a) * A.csf + c) * 4;
    const uint32_t kr = (uint32_t)v * 16u, ki = (uint32_t)A.kc + (uint32_t)v * 16u;
    const uint32_t ra = (uint32_t)a, rb = (uint32_t)(A.nant + a);
    P.st[r][0] = (kr >> 7) * region + sw128_offset(ra, kr & 127u);
    P.st[r][1] = (ki >> 7) * region + sw128_offset(ra, ki & 127u);
    P.st[r][2] = (kr >> 7) * region + sw128_offset(rb, kr & 127u);
    P.st[r][3] = (ki >> 7) * region + sw128_offset(rb, ki & 127u);
  }
  P.q_step = (long long)(A.kc / 4 / A.csf) * pkt;
  P.f_step = (long long)A.ppfv * pkt;
  P.s_step = A.csf * 4;
}

DSB_DEV void tc_load_planned(const TcArgs& A, const TcFillPlan& P, int g, int f, int s, int q,
                             uint4 (&w)[TC_PRE]) {
  const uint8_t* base = A.raw + (size_t)g * A.raw_g_stride + (long long)f * P.f_step +
                        (long long)s * P.s_step + (long long)q * P.q_step;
  const int n = A.nant * (A.kc / 16);
#pragma unroll
  for (int r = 0; r < TC_PRE; ++r)
    if (threadIdx.x + r * TC_THREADS < n)
      w[r] = __ldg(reinterpret_cast<const uint4*>(base + P.ld[r]));
}

DSB_DEV void tc_store_planned(const TcArgs& A, const TcFillPlan& P, uint8_t* st,
                              const uint4 (&w)[TC_PRE]) {
  const int n = A.nant * (A.kc / 16);
#pragma unroll
  for (int r = 0; r < TC_PRE; ++r) {
    if (threadIdx.x + r * TC_THREADS < n) {
      uint4 R, I, N;
      R.x = nib_lo_s8x4(w[r].x); R.y = nib_lo_s8x4(w[r].y);
      R.z = nib_lo_s8x4(w[r].z); R.w = nib_lo_s8x4(w[r].w);
      I.x = nib_hi_s8x4(w[r].x); I.y = nib_hi_s8x4(w[r].y);
      I.z = nib_hi_s8x4(w[r].z); I.w = nib_hi_s8x4(w[r].w);
      N.x = neg_s8x4(R.x); N.y = neg_s8x4(R.y); N.z = neg_s8x4(R.z); N.w = neg_s8x4(R.w);
      *reinterpret_cast<uint4*>(st + P.st[r][0]) = R;
      *reinterpret_cast<uint4*>(st + P.st[r][1]) = I;
      *reinterpret_cast<uint4*>(st + P.st[r][2]) = I;
      *reinterpret_cast<uint4*>(st + P.st[r][3]) = N;
    }
  }
}

// Unpack the words of tc_load into the operand stage (same layout as tc_fill).
DSB_DEV void tc_store(const TcArgs& A, uint8_t* st, const uint4 (&w)[TC_PRE]) {
  const int nv = A.kc / 16;
  const int kc = A.kc;
  const uint32_t region = (uint32_t)A.rows * 128u;
  const int nant = A.nant;
#pragma unroll
  for (int r = 0; r < TC_PRE; ++r) {
    const int idx = threadIdx.x + r * TC_THREADS;
    if (idx < nant * nv) {
      const int a = idx / nv, v = idx % nv;
      uint4 R, I, N;
      R.x = nib_lo_s8x4(w[r].x); R.y = nib_lo_s8x4(w[r].y);
      R.z = nib_lo_s8x4(w[r].z); R.w = nib_lo_s8x4(w[r].w);
      I.x = nib_hi_s8x4(w[r].x); I.y = nib_hi_s8x4(w[r].y);
      I.z = nib_hi_s8x4(w[r].z); I.w = nib_hi_s8x4(w[r].w);
      N.x = neg_s8x4(R.x); N.y = neg_s8x4(R.y); N.z = neg_s8x4(R.z); N.w = neg_s8x4(R.w);
      const uint32_t kr = (uint32_t)v * 16u, ki = (uint32_t)kc + (uint32_t)v * 16u;
      const uint32_t ra = (uint32_t)a, rb = (uint32_t)(nant + a);
      *reinterpret_cast<uint4*>(st + (kr >> 7) * region + sw128_offset(ra, kr & 127u)) = R;
      *reinterpret_cast<uint4*>(st + (ki >> 7) * region + sw128_offset(ra, ki & 127u)) = I;
      *reinterpret_cast<uint4*>(st + (kr >> 7) * region + sw128_offset(rb, kr & 127u)) = I;
      *reinterpret_cast<uint4*>(st + (ki >> 7) * region + sw128_offset(rb, ki & 127u)) = N;
    }
  }
}

// Convert one K chunk of one unit from packed int4 into the operand stage:
// rows [0, nant) = [R | I], rows [nant, 2 nant) = [I | -R] (K-major, SW128).
DSB_DEV void tc_fill(const TcArgs& A, uint8_t* st, int g, int f, int s, int q) {
  const int nw = A.kc / 4;  // 32-bit words (4 complex samples) per antenna per chunk
  const int kc = A.kc;
  const uint32_t region = (uint32_t)A.rows * 128u;
  const uint8_t* base = A.raw + (size_t)g * A.raw_g_stride;
  const int nant = A.nant;
  if ((A.csf & 3) == 0 && (A.nchan & 3) == 0) {
    const int nv = nw / 4;
    for (int idx = threadIdx.x; idx < nant * nv; idx += TC_THREADS) {
      const int a = idx / nv, v = idx % nv;
      const int j = q * nw + v * 4;
      const int p = j / A.csf, c = j % A.csf;
      const uint4 w = __ldg(reinterpret_cast<const uint4*>(
          base + ((((size_t)(f * A.ppfv + p) * nant + a) * A.nchan + (size_t)s * A.csf + c) * 4)));
      uint4 R, I, N;
      R.x = nib_lo_s8x4(w.x); R.y = nib_lo_s8x4(w.y); R.z = nib_lo_s8x4(w.z); R.w = nib_lo_s8x4(w.w);
      I.x = nib_hi_s8x4(w.x); I.y = nib_hi_s8x4(w.y); I.z = nib_hi_s8x4(w.z); I.w = nib_hi_s8x4(w.w);
      N.x = neg_s8x4(R.x); N.y = neg_s8x4(R.y); N.z = neg_s8x4(R.z); N.w = neg_s8x4(R.w);
      const uint32_t kr = (uint32_t)v * 16u, ki = (uint32_t)kc + (uint32_t)v * 16u;
      const uint32_t ra = (uint32_t)a, rb = (uint32_t)(nant + a);
      *reinterpret_cast<uint4*>(st + (kr >> 7) * region + sw128_offset(ra, kr & 127u)) = R;
      *reinterpret_cast<uint4*>(st + (ki >> 7) * region + sw128_offset(ra, ki & 127u)) = I;
      *reinterpret_cast<uint4*>(st + (kr >> 7) * region + sw128_offset(rb, kr & 127u)) = I;
      *reinterpret_cast<uint4*>(st + (ki >> 7) * region + sw128_offset(rb, ki & 127u)) = N;
    }
  } else {
    for (int idx = threadIdx.x; idx < nant * nw; idx += TC_THREADS) {
      const int a = idx / nw, jj = idx % nw;
      const int j = q * nw + jj;
      const int p = j / A.csf, c = j % A.csf;
      const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(
          base + ((((size_t)(f * A.ppfv + p) * nant + a) * A.nchan + (size_t)s * A.csf + c) * 4)));
      const uint32_t R = nib_lo_s8x4(w), I = nib_hi_s8x4(w), N = neg_s8x4(R);
      const uint32_t kr = (uint32_t)jj * 4u, ki = (uint32_t)kc + (uint32_t)jj * 4u;
      const uint32_t ra = (uint32_t)a, rb = (uint32_t)(nant + a);
      *reinterpret_cast<uint32_t*>(st + (kr >> 7) * region + sw128_offset(ra, kr & 127u)) = R;
      *reinterpret_cast<uint32_t*>(st + (ki >> 7) * region + sw128_offset(ra, ki & 127u)) = I;
      *reinterpret_cast<uint32_t*>(st + (kr >> 7) * region + sw128_offset(rb, kr & 127u)) = I;
      *reinterpret_cast<uint32_t*>(st + (ki >> 7) * region + sw128_offset(rb, ki & 127u)) = N;
    }
  }
}

// Read accumulator `buf` (rows b < nant; columns a: Re, nant + a: Im) and
// emit the upper triangle b <= a at bls(a, b) (conj(E_b) E_a).
// Warp w reads TMEM lane quarter (w & 3) (rows 32*(w&3) ...) and every
// other 16-column chunk (w >> 2 picks the parity).
// Shared copies of the gridding CSR of the (chgroup, subband) last used.
struct TcTab {
  int* roff;        // (TC_CAP_ROWS + 1) row offsets relative to the group's first entry
  uint16_t* bls;    // (nbase) baseline of each entry
  int* cached;      // group index whose tables are loaded (-1 none)
};

template <int MODE>
DSB_DEV void tc_epilogue(const TcArgs& A, uint32_t tmem_base, int buf, int g, int f, int s,
                         int2* vbuf, const TcTab& tab) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quarter = warp & 3, half = warp >> 2;
  const int nant = A.nant;
  const int b = quarter * 32 + lane;
  if (quarter * 32 < nant) {
    const uint32_t lane_base =
        tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * 256);
    for (int c0 = half * 16; c0 < nant; c0 += 32) {
      if (c0 + 15 < quarter * 32) continue;  // whole chunk below this warp's rows
      uint32_t vr[16], vi[16];
      tmem_ld16(lane_base + (uint32_t)c0, vr);
      tmem_ld16(lane_base + (uint32_t)(nant + c0), vi);
      tmem_ld_wait();
      if (b < nant) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int a = c0 + j;
          if (a < b || a >= nant) continue;
          const int bls = upper_bls(a, b);
          const int re = (int)vr[j], im = (int)vi[j];
          if constexpr (MODE == 0) {
            A.out[(size_t)g * A.o_g + (size_t)f * A.o_f + (size_t)bls * A.o_b + (size_t)s * A.o_s] =
                make_float2((float)re, (float)im);
          } else if (A.gains) {
            // calibrated: V' = g_a conj(g_b) V (V = conj(E_b) E_a), every
            // product and sum rounded on its own (no contraction)
            const float2* gs = A.gains + ((size_t)g * A.ceff + s) * nant;
            const float2 ga = gs[a], gb = gs[b];
            const float pr = __fadd_rn(__fmul_rn(ga.x, gb.x), __fmul_rn(ga.y, gb.y));
            const float pi = __fsub_rn(__fmul_rn(ga.y, gb.x), __fmul_rn(ga.x, gb.y));
            const float fr = (float)re, fi = (float)im;
            reinterpret_cast<float2*>(vbuf)[bls] =
                make_float2(__fsub_rn(__fmul_rn(fr, pr), __fmul_rn(fi, pi)),
                            __fadd_rn(__fmul_rn(fr, pi), __fmul_rn(fi, pr)));
          } else {
            vbuf[bls] = make_int2(re, im);
          }
        }
      }
    }
  }
  tc_fence_before();
  if constexpr (MODE == 1) {
    // per-cell sum over the baselines gridded into it (exact int32); the
    // group's CSR is copied to shared memory when the group changes (a CTA
    // walks consecutive tiles of one group)
    const int gs = g * A.ceff + s;
    const long long row0 = A.yoff[gs];
    const int cnt = A.ycnt[gs];
    const int e0 = A.row_off[row0];
    const int ne = A.row_off[row0 + cnt] - e0;
    const bool use_tab = cnt <= TC_CAP_ROWS && ne <= A.nant * (A.nant + 1) / 2;
    const bool reload = use_tab && *tab.cached != gs;
    if (reload) {
      for (int k = threadIdx.x; k <= cnt; k += TC_THREADS) tab.roff[k] = A.row_off[row0 + k] - e0;
      for (int j = threadIdx.x; j < ne; j += TC_THREADS) tab.bls[j] = (uint16_t)A.row_bls[e0 + j];
    }
    __syncthreads();
    if (reload && threadIdx.x == 0) *tab.cached = gs;
    const long long tp = (A.t_base + f) & A.t_mask;
    float2* yrow = A.yout + tp * A.y_t_stride + row0;
    if (cnt > 0 && !(DSB_INB(row0, A.y_t_stride, A.status) &&
                     DSB_INB(row0 + cnt - 1, A.y_t_stride, A.status)))
      return;
    if (A.gains) {
      // calibrated visibilities: float sums in CSR order
      const float2* fbuf = reinterpret_cast<const float2*>(vbuf);
      for (int k = threadIdx.x; k < cnt; k += TC_THREADS) {
        const long long r = row0 + k;
        float sr = 0.f, si = 0.f;
        const int j0 = use_tab ? tab.roff[k] + e0 : A.row_off[r];
        const int j1 = use_tab ? tab.roff[k + 1] + e0 : A.row_off[r + 1];
        for (int j = j0; j < j1; ++j) {
          const int bl = use_tab ? (int)tab.bls[j - e0] : A.row_bls[j];
          if (!DSB_INB(bl, A.nant * (A.nant + 1) / 2, A.status)) continue;
          sr = __fadd_rn(sr, fbuf[bl].x);
          si = __fadd_rn(si, fbuf[bl].y);
        }
        yrow[k] = make_float2(sr, si);
      }
    } else if (use_tab) {
      for (int k = threadIdx.x; k < cnt; k += TC_THREADS) {
        int sr = 0, si = 0;
        const int j1 = tab.roff[k + 1];
        for (int j = tab.roff[k]; j < j1; ++j) {
          if (!DSB_INB(tab.bls[j], A.nant * (A.nant + 1) / 2, A.status)) continue;
          const int2 v = vbuf[tab.bls[j]];
          sr += v.x;
          si += v.y;
        }
        yrow[k] = make_float2((float)sr, (float)si);
      }
    } else {
      for (int k = threadIdx.x; k < cnt; k += TC_THREADS) {
        const long long r = row0 + k;
        int sr = 0, si = 0;
        for (int j = A.row_off[r]; j < A.row_off[r + 1]; ++j) {
          if (!DSB_INB(A.row_bls[j], A.nant * (A.nant + 1) / 2, A.status)) continue;
          const int2 v = vbuf[A.row_bls[j]];
          sr += v.x;
          si += v.y;
        }
        yrow[k] = make_float2((float)sr, (float)si);
      }
    }
  }
}

template <int MODE, bool TMA>
__global__ void __launch_bounds__(TC_THREADS, 1)
    corr_tc_kernel(const TcArgs A, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* stages = smem;
  // TMA: nraw raw stages after the operand stages (both 1024-byte multiples)
  uint8_t* raw_st = stages + (size_t)A.nstage * A.stage_bytes;
  uint64_t* bar_mma =
      reinterpret_cast<uint64_t*>(raw_st + (TMA ? (size_t)A.nraw * A.raw_stage : 0));
  uint64_t* bar_acc = bar_mma + A.nstage;
  uint64_t* bar_drain = bar_acc + 2;
  uint64_t* bar_raw = bar_drain + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_raw + (TMA ? A.nraw : 0));
  int2* vbuf = reinterpret_cast<int2*>(tmem_slot + 4);
  TcTab tab{};
  if constexpr (MODE == 1) {
    tab.cached = reinterpret_cast<int*>(vbuf + A.nant * (A.nant + 1) / 2);
    tab.roff = tab.cached + 4;
    tab.bls = reinterpret_cast<uint16_t*>(tab.roff + TC_CAP_ROWS + 1);
  }

  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    tmem_alloc(tmem_slot, TC_TMEM_COLS);
    tmem_relinquish();
  }
  if (tid == 0) {
    if constexpr (MODE == 1) *tab.cached = -1;
    for (int i = 0; i < A.nstage; ++i) mbar_init(&bar_mma[i], 1);
    mbar_init(&bar_acc[0], 1);
    mbar_init(&bar_acc[1], 1);
    mbar_init(bar_drain, 1);
    if constexpr (TMA)
      for (int i = 0; i < A.nraw; ++i) mbar_init(&bar_raw[i], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  // each CTA walks a contiguous range of units (consecutive fast-vis tiles
  // of one (chgroup, subband) share the gridding tables)
  const int n_units = A.n_chgroup * A.n_fv * A.ceff;
  const int per_cta = (n_units + (int)gridDim.x - 1) / (int)gridDim.x;
  const int u_begin = (int)blockIdx.x * per_cta;
  const int my_units = max(0, min(per_cta, n_units - u_begin));
  const int n_items = my_units * A.n_chunks;
  const uint32_t idesc = idesc_i8(128u, (uint32_t)(2 * A.nant));
  const bool vec = (A.csf & 3) == 0 && (A.nchan & 3) == 0;
  const bool planned = vec && ((A.kc / 4) % A.csf) == 0;
  TcFillPlan plan{};
  if (planned) tc_fill_plan(A, plan);
  bool ok = true;
  // TMA: item `item`'s raw bytes (ppk packets x nant x csf channels x 4 bytes
  // of one chgroup page) into raw stage item % nraw, by thread 0
  int issued = 0, it_stop = n_items;
  auto issue_raw = [&](int item) {
    const int lu = item / A.n_chunks, q = item % A.n_chunks;
    int g, f, s;
    tc_unit_coords(A, u_begin + lu, g, f, s);
    const int r = item % A.nraw;
    mbar_arrive_expect_tx(&bar_raw[r], (uint32_t)(A.ppk * A.nant * A.csf * 4));
    tma_load_4d(raw_st + (size_t)r * A.raw_stage, &tmap, s * A.csf * 4, 0,
                f * A.ppfv + q * A.ppk, g, &bar_raw[r]);
  };
  if constexpr (TMA) {
    if (tid == 0)
      for (; issued < A.nraw - 1 && issued < n_items; ++issued) issue_raw(issued);
  }
  // the raw words of the next item are loaded while this one is unpacked
  uint4 pre[TC_PRE];
  if (!TMA && vec && n_items > 0) {
    int g0, f0, s0;
    tc_unit_coords(A, u_begin, g0, f0, s0);
    if (planned) tc_load_planned(A, plan, g0, f0, s0, 0, pre);
    else tc_load(A, g0, f0, s0, 0, pre);
  }

  for (int it = 0; it < n_items; ++it) {
    const int lu = it / A.n_chunks, q = it % A.n_chunks;
    const int u = u_begin + lu;
    int g, f, s;
    tc_unit_coords(A, u, g, f, s);
    const int slot = it % A.nstage;
    bool w_ok = true;
    if (it >= A.nstage) w_ok = mbar_wait(&bar_mma[slot], (uint32_t)((it / A.nstage - 1) & 1));
    if constexpr (TMA)
      w_ok = w_ok && mbar_wait(&bar_raw[it % A.nraw], (uint32_t)((it / A.nraw) & 1));
    if (!__syncthreads_and(w_ok)) { ok = false; it_stop = it; break; }
    uint8_t* st = stages + (size_t)slot * A.stage_bytes;
    if constexpr (TMA) {
      // every thread is done with item it - 1: its raw stage takes item
      // it + nraw - 1
      if (tid == 0 && issued < n_items) issue_raw(issued++);
      const uint8_t* rs = raw_st + (size_t)(it % A.nraw) * A.raw_stage;
      const int n_w = A.nant * (A.kc / 16);
      uint4 cur[TC_PRE];
#pragma unroll
      for (int r = 0; r < TC_PRE; ++r)
        if (tid + r * TC_THREADS < n_w) cur[r] = *reinterpret_cast<const uint4*>(rs + plan.lds[r]);
      tc_store_planned(A, plan, st, cur);
    } else if (vec) {
      uint4 cur[TC_PRE];
#pragma unroll
      for (int r = 0; r < TC_PRE; ++r) cur[r] = pre[r];
      if (it + 1 < n_items) {
        const int nlu = (it + 1) / A.n_chunks, nq = (it + 1) % A.n_chunks;
        int ng, nf, ns;
        tc_unit_coords(A, u_begin + nlu, ng, nf, ns);
        if (planned) tc_load_planned(A, plan, ng, nf, ns, nq, pre);
        else tc_load(A, ng, nf, ns, nq, pre);
      }
      if (planned) tc_store_planned(A, plan, st, cur);
      else tc_store(A, st, cur);
    } else {
      tc_fill(A, st, g, f, s, q);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t d = tmem_base + (uint32_t)((lu & 1) * 256);
      const uint32_t sbase = smem_u32(st);
      for (int m = 0; m < A.n_mma; ++m) {
        const uint32_t kb = (uint32_t)m * 32u;
        const uint64_t desc = sdesc_k_sw128(sbase + (kb >> 7) * (uint32_t)A.rows * 128u + (kb & 127u));
        umma_i8_ss(d, desc, desc, idesc, (q > 0 || m > 0) ? 1u : 0u);
      }
      umma_commit(&bar_mma[slot]);
      if (q == A.n_chunks - 1) umma_commit(&bar_acc[lu & 1]);
    }
    if (q == A.n_chunks - 1 && lu >= 1) {
      const int pl = lu - 1;
      const bool a_ok = mbar_wait(&bar_acc[pl & 1], (uint32_t)((pl >> 1) & 1));
      if (!__syncthreads_and(a_ok)) { ok = false; it_stop = it; break; }
      tc_fence_after();
      int pg, pf, ps;
      tc_unit_coords(A, u_begin + pl, pg, pf, ps);
      tc_epilogue<MODE>(A, tmem_base, pl & 1, pg, pf, ps, vbuf, tab);
    }
  }
  if (ok && my_units > 0) {
    const int pl = my_units - 1;
    const bool a_ok = mbar_wait(&bar_acc[pl & 1], (uint32_t)((pl >> 1) & 1));
    if (__syncthreads_and(a_ok)) {
      tc_fence_after();
      int pg, pf, ps;
      tc_unit_coords(A, u_begin + pl, pg, pf, ps);
      tc_epilogue<MODE>(A, tmem_base, pl & 1, pg, pf, ps, vbuf, tab);
    } else {
      ok = false;
    }
  }
  if (!ok) {
    if (tid == 0) dsb_flag(A.status, DSB_E_TIMEOUT);
    // Drain every MMA this CTA issued before releasing tensor memory, and
    // every tensor copy still writing into its shared memory.
    if (tid == 0) {
      umma_commit(bar_drain);
      mbar_wait(bar_drain, 0u);
      if constexpr (TMA)
        for (int i = it_stop; i < issued; ++i)
          mbar_wait(&bar_raw[i % A.nraw], (uint32_t)((i / A.nraw) & 1));
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TC_TMEM_COLS);
  }
}

// ===========================================================================
// tensor-core correlator on split (GEMM-layout) voltages: tcgen05 kind::f16
// (int8 codes and float16 voltages, exact conversion to f16) or kind::tf32
// (float32 voltages, rounded to tf32 as a float32 tensor-core product does),
// float32 accumulators in TMEM.
// ===========================================================================
struct SplitTcArgs {
  const void* re;
  const void* im;
  int dtype;                 // DSB_DT_INT8 / DSB_DT_F16 / DSB_DT_F32
  int nchan, npkt, nant, nant_p, ppfv, fuse, csf, ceff;
  int n_fv, n_units, kprime, n_chunks, rows, nstage, stage_bytes;
  float2* out;
  int* status;
};

// Output unit u -> the fast-vis tile, its channel range and pols, and the
// output column: Stokes-I unit = (fv, summed channel s), K over (channel of
// the group, pol, t-sub, packet); 2-pol unit = (fv, ch, pol), K over
// (t-sub, packet).
DSB_DEV void split_unit(const SplitTcArgs& A, int u, int& fv, int& ch0, int& pol0, int& npol_u) {
  if (A.fuse) {
    fv = u / A.ceff;
    ch0 = (u % A.ceff) * A.csf;
    pol0 = 0;
    npol_u = 2;
  } else {
    fv = u / (A.nchan * 2);
    ch0 = (u / 2) % A.nchan;
    pol0 = u % 2;
    npol_u = 1;
  }
}

template <int ELEM>
DSB_DEV uint32_t split_load_bits(const SplitTcArgs& A, const void* p, size_t o) {
  if constexpr (ELEM == 2) {
    if (A.dtype == DSB_DT_INT8)
      return (uint32_t)__half_as_ushort(__int2half_rn((int)static_cast<const int8_t*>(p)[o]));
    return (uint32_t)__half_as_ushort(static_cast<const __half*>(p)[o]);
  } else {
    // round the float32 to tf32 (10 mantissa bits), nearest with ties away
    // from zero: add half of the dropped range to the magnitude bits (a
    // carry moves into the exponent correctly), clear the dropped bits;
    // infinities and NaNs pass unchanged
    const uint32_t u = __float_as_uint(static_cast<const float*>(p)[o]);
    if ((u & 0x7F800000u) == 0x7F800000u) return u;
    return (u + 0x1000u) & 0xFFFFE000u;
  }
}

// One K chunk (KC complex samples) of unit u into an operand stage:
// rows [0, nant_p) = [R | I], rows [nant_p, 2 nant_p) = [I | -R] (K-major,
// SW128, one 128-byte row per operand row); samples past the unit's K and
// antennas past nant are zero.
template <int ELEM>
DSB_DEV void split_fill(const SplitTcArgs& A, uint8_t* st, int u, int q) {
  constexpr int KC = 64 / ELEM;    // complex samples per chunk
  constexpr int G = 16 / ELEM;     // samples per 16-byte group
  constexpr int NG = KC / G;       // groups per half row (4)
  int fv, ch0, pol0, npol_u;
  split_unit(A, u, fv, ch0, pol0, npol_u);
  const size_t plane = (size_t)A.npkt * A.nant;
  for (int idx = threadIdx.x; idx < A.nant_p * NG; idx += TC_THREADS) {
    const int a = idx % A.nant_p, j = idx / A.nant_p;
    uint32_t r[G], m[G];
#pragma unroll
    for (int i = 0; i < G; ++i) {
      int k = q * KC + j * G + i;
      r[i] = 0u;
      m[i] = 0u;
      if (a < A.nant && k < A.kprime) {
        const int p = k % A.ppfv;
        k /= A.ppfv;
        const int t = k & 1;
        k >>= 1;
        const int pol = pol0 + k % npol_u;
        const int ch = ch0 + k / npol_u;
        const size_t o = (((size_t)ch * 2 + t) * 2 + pol) * plane +
                         (size_t)(fv * A.ppfv + p) * A.nant + a;
        r[i] = split_load_bits<ELEM>(A, A.re, o);
        m[i] = split_load_bits<ELEM>(A, A.im, o);
      }
    }
    uint4 R, I, N;
    if constexpr (ELEM == 2) {
      R = make_uint4(r[0] | (r[1] << 16), r[2] | (r[3] << 16), r[4] | (r[5] << 16),
                     r[6] | (r[7] << 16));
      I = make_uint4(m[0] | (m[1] << 16), m[2] | (m[3] << 16), m[4] | (m[5] << 16),
                     m[6] | (m[7] << 16));
      N = make_uint4(R.x ^ 0x80008000u, R.y ^ 0x80008000u, R.z ^ 0x80008000u,
                     R.w ^ 0x80008000u);
    } else {
      R = make_uint4(r[0], r[1], r[2], r[3]);
      I = make_uint4(m[0], m[1], m[2], m[3]);
      N = make_uint4(r[0] ^ 0x80000000u, r[1] ^ 0x80000000u, r[2] ^ 0x80000000u,
                     r[3] ^ 0x80000000u);
    }
    const uint32_t kr = (uint32_t)j * 16u, ki = 64u + (uint32_t)j * 16u;
    const uint32_t ra = (uint32_t)a, rb = (uint32_t)(A.nant_p + a);
    *reinterpret_cast<uint4*>(st + sw128_offset(ra, kr)) = R;
    *reinterpret_cast<uint4*>(st + sw128_offset(ra, ki)) = I;
    *reinterpret_cast<uint4*>(st + sw128_offset(rb, kr)) = I;
    *reinterpret_cast<uint4*>(st + sw128_offset(rb, ki)) = N;
  }
}

// Accumulator `buf` of unit u: rows b < nant, columns a (Re) and nant_p + a
// (Im); the upper triangle b <= a goes to bls(a, b) (conj(E_b) E_a).
DSB_DEV void split_epilogue(const SplitTcArgs& A, uint32_t tmem_base, int buf, int u) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quarter = warp & 3, half = warp >> 2;
  const int nant = A.nant, nbase = nant * (nant + 1) / 2;
  const int b = quarter * 32 + lane;
  int fv, ch0, pol0, npol_u;
  split_unit(A, u, fv, ch0, pol0, npol_u);
  if (quarter * 32 < nant) {
    const uint32_t lane_base =
        tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * 256);
    for (int c0 = half * 16; c0 < nant; c0 += 32) {
      if (c0 + 15 < quarter * 32) continue;  // whole chunk below this warp's rows
      uint32_t vr[16], vi[16];
      tmem_ld16(lane_base + (uint32_t)c0, vr);
      tmem_ld16(lane_base + (uint32_t)(A.nant_p + c0), vi);
      tmem_ld_wait();
      if (b < nant) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int a = c0 + j;
          if (a < b || a >= nant) continue;
          const size_t bls = (size_t)upper_bls(a, b);
          const size_t o = A.fuse ? ((size_t)fv * nbase + bls) * A.ceff + ch0 / A.csf
                                  : (((size_t)fv * nbase + bls) * A.nchan + ch0) * 2 + pol0;
          A.out[o] = make_float2(__uint_as_float(vr[j]), __uint_as_float(vi[j]));
        }
      }
    }
  }
}

template <int ELEM>
__global__ void __launch_bounds__(TC_THREADS, 1) corr_split_tc_kernel(const SplitTcArgs A) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* stages = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bar_mma = reinterpret_cast<uint64_t*>(stages + (size_t)A.nstage * A.stage_bytes);
  uint64_t* bar_acc = bar_mma + A.nstage;
  uint64_t* bar_drain = bar_acc + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_drain + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    tmem_alloc(tmem_slot, TC_TMEM_COLS);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < A.nstage; ++i) mbar_init(&bar_mma[i], 1);
    mbar_init(&bar_acc[0], 1);
    mbar_init(&bar_acc[1], 1);
    mbar_init(bar_drain, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const int per_cta = (A.n_units + (int)gridDim.x - 1) / (int)gridDim.x;
  const int u_begin = (int)blockIdx.x * per_cta;
  const int my_units = max(0, min(per_cta, A.n_units - u_begin));
  const int n_items = my_units * A.n_chunks;
  // c_format F32; a/b format F16 (0) or TF32 (2); K-major; N = 2 nant_p; M = 128
  constexpr uint32_t fmt = ELEM == 2 ? 0u : 2u;
  const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) |
                         (((uint32_t)(2 * A.nant_p) >> 3) << 17) | ((128u >> 4) << 24);
  bool ok = true;
  for (int it = 0; it < n_items; ++it) {
    const int lu = it / A.n_chunks, q = it % A.n_chunks;
    const int slot = it % A.nstage;
    bool w_ok = true;
    if (it >= A.nstage) w_ok = mbar_wait(&bar_mma[slot], (uint32_t)((it / A.nstage - 1) & 1));
    if (!__syncthreads_and(w_ok)) { ok = false; break; }
    uint8_t* st = stages + (size_t)slot * A.stage_bytes;
    split_fill<ELEM>(A, st, u_begin + lu, q);
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t d = tmem_base + (uint32_t)((lu & 1) * 256);
      const uint32_t sbase = smem_u32(st);
#pragma unroll
      for (int m = 0; m < 4; ++m) {   // 4 MMAs of 32 bytes of K each
        const uint64_t desc = sdesc_k_sw128(sbase + (uint32_t)m * 32u);
        if constexpr (ELEM == 2) umma_f16_ss(d, desc, desc, idesc, (q > 0 || m > 0) ? 1u : 0u);
        else umma_tf32_ss(d, desc, desc, idesc, (q > 0 || m > 0) ? 1u : 0u);
      }
      umma_commit(&bar_mma[slot]);
      if (q == A.n_chunks - 1) umma_commit(&bar_acc[lu & 1]);
    }
    if (q == A.n_chunks - 1 && lu >= 1) {
      const int pl = lu - 1;
      const bool a_ok = mbar_wait(&bar_acc[pl & 1], (uint32_t)((pl >> 1) & 1));
      if (!__syncthreads_and(a_ok)) { ok = false; break; }
      tc_fence_after();
      split_epilogue(A, tmem_base, pl & 1, u_begin + pl);
      tc_fence_before();
    }
  }
  if (ok && my_units > 0) {
    const int pl = my_units - 1;
    const bool a_ok = mbar_wait(&bar_acc[pl & 1], (uint32_t)((pl >> 1) & 1));
    if (__syncthreads_and(a_ok)) {
      tc_fence_after();
      split_epilogue(A, tmem_base, pl & 1, u_begin + pl);
    } else {
      ok = false;
    }
  }
  if (!ok && tid == 0) {
    dsb_flag(A.status, DSB_E_TIMEOUT);
    // drain every MMA this CTA issued before tensor memory is released
    umma_commit(bar_drain);
    mbar_wait(bar_drain, 0u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TC_TMEM_COLS);
  }
}

int g_num_sms = 0;
int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DSB_OK : DSB_E_CUDA;
}

// Shared memory beyond the operand stages: mode 1 keeps the upper-triangle
// visibilities of one unit (int2) and the gridding tables of one group.
int tc_extra_bytes(const TcArgs& A, int mode) {
  if (mode != 1) return 0;
  const int nbase = A.nant * (A.nant + 1) / 2;
  return nbase * 8 + 16 + (TC_CAP_ROWS + 1) * 4 + nbase * 2 + 16;
}

// Fill the derived geometry; returns DSB_OK or an error code.
int tc_plan(TcArgs& A, int mode) {
  if (A.nant < 16 || A.nant > 128 || (A.nant % 16) != 0) return DSB_E_UNSUPPORTED;
  if (A.t_int <= 0 || (A.t_int % 2) != 0 || A.npkt % (A.t_int / 2) != 0) return DSB_E_ARG;
  if (A.csf <= 0 || A.nchan % A.csf != 0) return DSB_E_ARG;
  A.ppfv = A.t_int / 2;
  A.n_fv = A.npkt / A.ppfv;
  A.ceff = A.nchan / A.csf;
  const int kprime = 2 * A.t_int * A.csf;  // complex samples per antenna per unit
  if (kprime % 16 != 0) return DSB_E_UNSUPPORTED;
  A.kc = std::min(kprime, 128);
  while (kprime % A.kc != 0) A.kc -= 16;
  A.n_chunks = kprime / A.kc;
  A.rows = std::max(128, ((2 * A.nant + 7) / 8) * 8);
  A.nkblk = (2 * A.kc + 127) / 128;
  A.stage_bytes = A.nkblk * A.rows * 128;
  A.n_mma = 2 * A.kc / 32;
  const int extra = tc_extra_bytes(A, mode);
  const int budget = TC_SMEM_BUDGET - extra - 1024 - 256;
  A.nstage = std::min(4, budget / A.stage_bytes);
  if (A.nstage < 2) return DSB_E_UNSUPPORTED;
  // raw staging by TMA when a chunk is whole packets of 16-byte channel runs
  // and four raw stages still leave two operand stages
  A.tma = 0;
  if ((A.csf % 4) == 0 && (A.nchan % 4) == 0 && ((A.kc / 4) % A.csf) == 0 && A.nant <= 256) {
    A.ppk = (A.kc / 4) / A.csf;
    A.raw_stage = (A.ppk * A.nant * A.csf * 4 + 1023) & ~1023;
    A.nraw = 4;
    const int ns = std::min(4, (budget - A.nraw * A.raw_stage) / A.stage_bytes);
    if (ns >= 2) {
      A.tma = 1;
      A.nstage = ns;
    }
  }
  return DSB_OK;
}

// The driver's tensor-map encoder, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  }
  return fn;
}

// The raw pages as a 4-D uint8 tensor (channel bytes, antenna, packet,
// chgroup) with one item's box (csf channels x 4 bytes, every antenna, ppk
// packets, one chgroup).  False if it cannot be encoded (the kernel then
// loads the raw words itself).
bool tc_raw_tmap(const TcArgs& A, CUtensorMap* m) {
  auto fn = tmap_encoder();
  if (!fn) return false;
  const cuuint64_t row = (cuuint64_t)A.nchan * 4;
  const cuuint64_t pkt = row * (cuuint64_t)A.nant;
  const cuuint64_t gs = A.n_chgroup > 1 ? (cuuint64_t)A.raw_g_stride : pkt * (cuuint64_t)A.npkt;
  const cuuint64_t dims[4] = {row, (cuuint64_t)A.nant, (cuuint64_t)A.npkt,
                              (cuuint64_t)A.n_chgroup};
  const cuuint64_t strides[3] = {row, pkt, gs};
  const cuuint32_t box[4] = {(cuuint32_t)(A.csf * 4), (cuuint32_t)A.nant, (cuuint32_t)A.ppk, 1u};
  const cuuint32_t es[4] = {1u, 1u, 1u, 1u};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<uint8_t*>(A.raw), dims, strides, box,
            es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_64B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Launch corr_tc_kernel<MODE, TMA> on the planned geometry.
template <int MODE>
int tc_launch(TcArgs& A, int grid, cudaStream_t stream) {
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  if (A.tma && !tc_raw_tmap(A, &tmap)) A.tma = 0;
  const int raw = A.tma ? A.nraw * A.raw_stage : 0;
  const int smem = std::max(A.nstage * A.stage_bytes + raw + 1024 + 256 + tc_extra_bytes(A, MODE),
                            TC_MIN_SMEM);
  if (A.tma) {
    cudaFuncSetAttribute(corr_tc_kernel<MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem);
    corr_tc_kernel<MODE, true><<<grid, TC_THREADS, smem, stream>>>(A, tmap);
  } else {
    cudaFuncSetAttribute(corr_tc_kernel<MODE, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    corr_tc_kernel<MODE, false><<<grid, TC_THREADS, smem, stream>>>(A, tmap);
  }
  return launch_status();
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int dsb_version(void) { return DSB_VERSION; }

const char* dsb_strerror(int code) {
  switch (code) {
    case DSB_OK: return "ok";
    case DSB_E_ARG: return "invalid argument";
    case DSB_E_CUDA: return "CUDA runtime error";
    case DSB_E_UNSUPPORTED: return "unsupported geometry";
    case DSB_E_TIMEOUT: return "device-side bounded wait ran out";
    case DSB_E_CAPACITY: return "size exceeds a fixed capacity";
    case DSB_E_BOUNDS: return "index out of range (bounds-checked build)";
    default: return "unknown error";
  }
}

int dsb_unpack_int4(const void* raw, int npkt, int nant, int nchan, int out_dtype, float scale,
                    void* out_re, void* out_im, cudaStream_t stream) {
  if (!raw || !out_re || !out_im || npkt <= 0 || nant <= 0 || nchan <= 0) return DSB_E_ARG;
  const int rows = npkt * nant;
  dim3 grid((rows + 31) / 32, (nchan + 31) / 32), block(32, 8);
  const uint32_t* r = static_cast<const uint32_t*>(raw);
  switch (out_dtype) {
    case DSB_DT_INT8:
      unpack_kernel<int8_t><<<grid, block, 0, stream>>>(r, rows, nchan, scale, (int8_t*)out_re,
                                                        (int8_t*)out_im);
      break;
    case DSB_DT_F16:
      unpack_kernel<__half><<<grid, block, 0, stream>>>(r, rows, nchan, scale, (__half*)out_re,
                                                        (__half*)out_im);
      break;
    case DSB_DT_F32:
      unpack_kernel<float><<<grid, block, 0, stream>>>(r, rows, nchan, scale, (float*)out_re,
                                                       (float*)out_im);
      break;
    default: return DSB_E_ARG;
  }
  return launch_status();
}

int dsb_corr_split(const void* re, const void* im, int in_dtype, int nchan, int npkt, int nant,
                   int t_int, int fuse_stokes_i, int csf, void* out, int* status,
                   cudaStream_t stream) {
  if (!re || !im || !out || nchan <= 0 || npkt <= 0 || nant <= 0) return DSB_E_ARG;
  if (t_int <= 0 || t_int % 2 || npkt % (t_int / 2)) return DSB_E_ARG;
  if (nant > 128) return DSB_E_UNSUPPORTED;
  if (in_dtype != DSB_DT_INT8 && in_dtype != DSB_DT_F16 && in_dtype != DSB_DT_F32)
    return DSB_E_ARG;
  SplitTcArgs A{};
  A.re = re; A.im = im; A.dtype = in_dtype;
  A.nchan = nchan; A.npkt = npkt; A.nant = nant;
  A.nant_p = (nant + 7) & ~7;
  A.ppfv = t_int / 2;
  A.n_fv = npkt / A.ppfv;
  A.fuse = fuse_stokes_i ? 1 : 0;
  if (A.fuse) {
    if (csf <= 0 || nchan % csf) return DSB_E_ARG;
    A.csf = csf;
    A.ceff = nchan / csf;
    A.n_units = A.n_fv * A.ceff;
    A.kprime = 2 * csf * t_int;     // (channel, pol, t-sub, packet)
  } else {
    A.csf = 1;
    A.ceff = nchan;
    A.n_units = A.n_fv * nchan * 2;
    A.kprime = t_int;               // (t-sub, packet)
  }
  const int kc = in_dtype == DSB_DT_F32 ? 16 : 32;
  A.n_chunks = (A.kprime + kc - 1) / kc;
  A.rows = std::max(128, 2 * A.nant_p);
  A.stage_bytes = A.rows * 128;
  A.nstage = 4;
  A.out = static_cast<float2*>(out);
  A.status = status;
  const int smem = A.nstage * A.stage_bytes + 1024 + (A.nstage + 3) * 8 + 16;
  const int grid = std::min(A.n_units, num_sms());
  if (in_dtype == DSB_DT_F32) {
    cudaFuncSetAttribute(corr_split_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem);
    corr_split_tc_kernel<4><<<grid, TC_THREADS, smem, stream>>>(A);
  } else {
    cudaFuncSetAttribute(corr_split_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem);
    corr_split_tc_kernel<2><<<grid, TC_THREADS, smem, stream>>>(A);
  }
  return launch_status();
}

int dsb_corr_tc(const void* raw, long long raw_g_stride, int n_chgroup, int npkt, int nant,
                int nchan, int t_int, int csf, int unit_order, void* out, long long o_g,
                long long o_f, long long o_b, long long o_s, int max_ctas, int* status,
                cudaStream_t stream) {
  if (!raw || !out || n_chgroup <= 0 || npkt <= 0) return DSB_E_ARG;
  if (((uintptr_t)raw & 15) || (raw_g_stride & 15)) return DSB_E_ARG;
  TcArgs A{};
  A.raw = static_cast<const uint8_t*>(raw);
  A.raw_g_stride = raw_g_stride;
  A.n_chgroup = n_chgroup; A.npkt = npkt; A.nant = nant; A.nchan = nchan;
  A.t_int = t_int; A.csf = csf; A.unit_order = unit_order;
  A.out = static_cast<float2*>(out);
  A.o_g = o_g; A.o_f = o_f; A.o_b = o_b; A.o_s = o_s;
  A.status = status;
  int rc = tc_plan(A, 0);
  if (rc) return rc;
  const int n_units = n_chgroup * A.n_fv * A.ceff;
  return tc_launch<0>(A, std::min(n_units, max_ctas > 0 ? max_ctas : num_sms()), stream);
}

int dsb_corr_tc_grid(const void* raw, long long raw_g_stride, int n_chgroup, int npkt, int nant,
                     int nchan, int t_int, int csf, const int* yoff, const int* ycnt,
                     const int* row_off, const int* row_bls, void* yout, long long y_t_stride,
                     long long t_base, long long t_mask, int max_ctas, const void* gains,
                     int* status, cudaStream_t stream) {
  if (!raw || !yout || !yoff || !ycnt || !row_off || !row_bls) return DSB_E_ARG;
  if (((uintptr_t)raw & 15) || (raw_g_stride & 15)) return DSB_E_ARG;
  TcArgs A{};
  A.raw = static_cast<const uint8_t*>(raw);
  A.raw_g_stride = raw_g_stride;
  A.n_chgroup = n_chgroup; A.npkt = npkt; A.nant = nant; A.nchan = nchan;
  A.t_int = t_int; A.csf = csf; A.unit_order = 0;
  A.yoff = yoff; A.ycnt = ycnt; A.row_off = row_off; A.row_bls = row_bls;
  A.yout = static_cast<float2*>(yout);
  A.y_t_stride = y_t_stride; A.t_base = t_base; A.t_mask = t_mask;
  A.gains = static_cast<const float2*>(gains);
  A.status = status;
  int rc = tc_plan(A, 1);
  if (rc) return rc;
  const int n_units = n_chgroup * A.n_fv * A.ceff;
  return tc_launch<1>(A, std::min(n_units, max_ctas > 0 ? max_ctas : num_sms()), stream);
}

}  // extern "C"
