// Fused fine-DM combine + 2-D inverse real FFT (sm_100a).
//
// One image per (fine DM f, time t):
//   G_h[u, w] = 0.5 * sum_e s_e(D[t - sf[f, g_e]][row_e]) * (-1)^(u+w),  w in [0, N/2]
//   img[x, y] = irfft2(G_h)[x, y]        (1/N^2 normalisation, numpy/torch "backward")
// which replaces fused_dequant_combine_per_fdm_half + torch.fft.irfft2
// (src/dsart/image/fused_combine_cuda.py:560-620, image/imager_gpu.py:590).
//
// One CTA owns one image at a time (persistent loop over images); nothing
// but the ring reads and the image writes leaves the SM:
//
//  1. Combine.  The non-zero half-spectrum cells S (the union of every
//     chgroup's uv pattern, a few thousand cells) are summed in shared memory
//     from the time-major stage-2 ring: one coalesced read of each chgroup's
//     coarse-DM slice, shared-memory int32 atomics into S held in fixed
//     point (S * 2^k, k from a bound on the image's parts).  Each thread then
//     moves its own range of S (at most MAXE entries, whole slots) into
//     tensor memory, which this kernel uses as plain per-thread storage:
//     TMEM is otherwise idle here and holds S across the passes below while
//     the shared buffer is reused for the transforms.
//  2. Column transforms by decimation in frequency.  Columns w = 0 and N/2
//     of G_h are Hermitian in u, so their transforms are real: they ride
//     together as one complex column (w = 0 + i * w = N/2), leaving N/2
//     complex columns.  With N = FOLD * LC, output rows x = FOLD*m + p are
//         A[FOLD m + p, w] = sum_n' W_LC^(n' m) W_N^(n' p)
//                              sum_q i^(q p) G_h[n' + LC q, w]      (FOLD = 4)
//     so pass p (p = 0..3) folds S (read back from TMEM) into the occupied
//     slots (n', w) of a shared LC x N/2 complex buffer (66 KB for N = 256,
//     small enough for three CTAs per SM) and transforms its columns in
//     place.  A column whose entries all sit at n' = 0 transforms to a
//     constant, so it is broadcast instead (for the bench's array, half of
//     the columns); a column without entries is zero.
//  3. Row transforms of the pass's LC rows, two real rows per complex
//     transform (x_a + i x_b), staged in shared memory and written as float4.
//
// Every transform of length L = R*R runs on a group of R threads: an R-point
// DFT in registers, the twiddles W_L^(j*x1), one XOR-swizzled shared-memory
// transpose, and a second R-point DFT (the classic two-step factorisation).
// The shared-memory atomics of step 1 add integers, so an image does not
// depend on the order in which they land: it is the same from run to run.
#include "dsb_common.cuh"

#include <algorithm>
#include <type_traits>

namespace {

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

// Complex add / subtract as one packed float32-pair instruction.  Against
// two scalar adds this took the image kernel from 896 to 863 ms per block at
// the bench workload (the transforms are mostly butterflies).
DSB_DEV float2 cadd(float2 a, float2 b) { return f2_add(a, b); }
DSB_DEV float2 csub(float2 a, float2 b) { return f2_sub(a, b); }
DSB_DEV float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
DSB_DEV float2 cmul_i(float2 a) { return make_float2(-a.y, a.x); }  // i * a

// a * i^k for a k known only at run time, without branches: swap the parts
// for odd k, then flip the signs ((k+1) & 2 on the first, k & 2 on the second)
DSB_DEV float2 crot_rt(float2 a, unsigned k) {
  const bool sw = k & 1u;
  const float u = sw ? a.y : a.x, v = sw ? a.x : a.y;
  return make_float2(__uint_as_float(__float_as_uint(u) ^ (((k + 1u) & 2u) << 30)),
                     __uint_as_float(__float_as_uint(v) ^ ((k & 2u) << 30)));
}

// cos/sin of multiples of pi/8 (exact mathematical constants, float-rounded)
constexpr float C8 = 0.92387953251128674f;   // cos(pi/8)
constexpr float S8 = 0.38268343236508977f;   // sin(pi/8)
constexpr float R2 = 0.70710678118654752f;   // cos(pi/4)

// Inverse 4-point DFT, X[m] = sum_k a[k] i^(k m), in place (natural order).
DSB_DEV void idft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
  const float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, cmul_i(d13));
  a3 = csub(d02, cmul_i(d13));
}

// Inverse 8-point DFT (w = e^{+2 pi i/8}), natural order out.
DSB_DEV void idft8(float2 (&a)[8]) {
  // k = k1 + 2 k2: 4-point over k2 for k1 = 0, 1 -> C[k1][m2] at a[k1 + 2 m2]
  idft4(a[0], a[2], a[4], a[6]);
  idft4(a[1], a[3], a[5], a[7]);
  // twiddle C[1][m2] *= w8^m2
  a[3] = cmul(a[3], make_float2(R2, R2));
  a[5] = cmul_i(a[5]);
  a[7] = cmul(a[7], make_float2(-R2, R2));
  // X[m2 + 4 m1] = C[0][m2] + (-1)^m1 C[1][m2]
  float2 x[8];
#pragma unroll
  for (int m2 = 0; m2 < 4; ++m2) {
    x[m2] = cadd(a[2 * m2], a[2 * m2 + 1]);
    x[m2 + 4] = csub(a[2 * m2], a[2 * m2 + 1]);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = x[i];
}

// Inverse 16-point DFT (w = e^{+2 pi i/16}), natural order out.
DSB_DEV void idft16(float2 (&a)[16]) {
  // k = k1 + 4 k2: 4-point over k2 for each k1 -> C[k1][m2] at a[k1 + 4 m2]
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) idft4(a[k1], a[k1 + 4], a[k1 + 8], a[k1 + 12]);
  // twiddles w16^(k1 m2)
  a[5] = cmul(a[5], make_float2(C8, S8));     // k1=1, m2=1: e=1
  a[9] = cmul(a[9], make_float2(R2, R2));     // k1=1, m2=2: e=2
  a[13] = cmul(a[13], make_float2(S8, C8));   // k1=1, m2=3: e=3
  a[6] = cmul(a[6], make_float2(R2, R2));     // k1=2, m2=1: e=2
  a[10] = cmul_i(a[10]);                      // k1=2, m2=2: e=4
  a[14] = cmul(a[14], make_float2(-R2, R2));  // k1=2, m2=3: e=6
  a[7] = cmul(a[7], make_float2(S8, C8));     // k1=3, m2=1: e=3
  a[11] = cmul(a[11], make_float2(-R2, R2));  // k1=3, m2=2: e=6
  a[15] = cmul(a[15], make_float2(-C8, -S8)); // k1=3, m2=3: e=9
  // 4-point over k1 for each m2: X[m2 + 4 m1] from a[4 m2 + k1]
#pragma unroll
  for (int m2 = 0; m2 < 4; ++m2) idft4(a[4 * m2], a[4 * m2 + 1], a[4 * m2 + 2], a[4 * m2 + 3]);
  float2 x[16];
#pragma unroll
  for (int m2 = 0; m2 < 4; ++m2)
#pragma unroll
    for (int m1 = 0; m1 < 4; ++m1) x[m2 + 4 * m1] = a[4 * m2 + m1];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = x[i];
}

// W_32^j = exp(+2 pi i j / 32), j = 0..15 (cos and sin of j pi / 16, exact
// mathematical values rounded to float)
__device__ __constant__ float2 kW32[16] = {
    {1.0f, 0.0f},
    {0.98078528040323043f, 0.19509032201612825f},
    {0.92387953251128674f, 0.38268343236508978f},
    {0.83146961230254524f, 0.55557023301960218f},
    {0.70710678118654752f, 0.70710678118654752f},
    {0.55557023301960218f, 0.83146961230254524f},
    {0.38268343236508978f, 0.92387953251128674f},
    {0.19509032201612825f, 0.98078528040323043f},
    {0.0f, 1.0f},
    {-0.19509032201612825f, 0.98078528040323043f},
    {-0.38268343236508978f, 0.92387953251128674f},
    {-0.55557023301960218f, 0.83146961230254524f},
    {-0.70710678118654752f, 0.70710678118654752f},
    {-0.83146961230254524f, 0.55557023301960218f},
    {-0.92387953251128674f, 0.38268343236508978f},
    {-0.98078528040323043f, 0.19509032201612825f}};

// Inverse 32-point DFT, natural order out: two 16-point transforms of the
// even and odd samples, then one radix-2 stage with the twiddles W_32^m.
DSB_DEV void idft32(float2 (&a)[32]) {
  float2 e[16], o[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    e[k] = a[2 * k];
    o[k] = a[2 * k + 1];
  }
  idft16(e);
  idft16(o);
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const float2 t = m ? cmul(o[m], kW32[m]) : o[m];
    a[m] = cadd(e[m], t);
    a[m + 16] = csub(e[m], t);
  }
}

template <int R>
DSB_DEV void idftR(float2 (&a)[R]) {
  if constexpr (R == 32) idft32(a);
  else if constexpr (R == 16) idft16(a);
  else if constexpr (R == 8) idft8(a);
  else idft4(a[0], a[1], a[2], a[3]);
}

// a * W_8 = a * (1 + i) / sqrt(2)
DSB_DEV float2 cmul_w8(float2 a) { return make_float2(R2 * (a.x - a.y), R2 * (a.x + a.y)); }

// Stage-2 ring elements (FMT): 0 complex64; 1 the BF16 storage form (bf16
// re/im pairs in 32 bits); 2 the cint8 wire form (int8 re/im pairs in 16
// bits, value = the row's scale x q).  Decoded to float32 and multiplied by
// the slice's factor sc (a power of two for forms 0 and 1, the row's scale
// times one for form 2); T2 holds two adjacent cells (one 4-, 8- or 16-byte
// load).
template <int FMT> struct RingElem {
  using T = float2;
  using T2 = float4;
  static DSB_DEV T2 zero2() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  static DSB_DEV float2 lo(T2 w, float sc) { return make_float2(w.x * sc, w.y * sc); }
  static DSB_DEV float2 hi(T2 w, float sc) { return make_float2(w.z * sc, w.w * sc); }
  static DSB_DEV float2 get(const T* p, float sc) {
    const float2 v = *p;
    return make_float2(v.x * sc, v.y * sc);
  }
};
template <> struct RingElem<1> {
  using T = uint32_t;
  using T2 = uint2;
  static DSB_DEV float2 f(uint32_t w, float sc) {
    const float2 v = bf16_pair_to_f2(w);
    return make_float2(v.x * sc, v.y * sc);
  }
  static DSB_DEV T2 zero2() { return make_uint2(0u, 0u); }
  static DSB_DEV float2 lo(T2 w, float sc) { return f(w.x, sc); }
  static DSB_DEV float2 hi(T2 w, float sc) { return f(w.y, sc); }
  static DSB_DEV float2 get(const T* p, float sc) { return f(*p, sc); }
};
template <> struct RingElem<2> {
  using T = uint16_t;
  using T2 = uint32_t;
  static DSB_DEV float s8(uint32_t w, int b) { return (float)(int)(int8_t)(uint8_t)(w >> (8 * b)); }
  static DSB_DEV T2 zero2() { return 0u; }
  static DSB_DEV float2 lo(T2 w, float sc) { return make_float2(sc * s8(w, 0), sc * s8(w, 1)); }
  static DSB_DEV float2 hi(T2 w, float sc) { return make_float2(sc * s8(w, 2), sc * s8(w, 3)); }
  static DSB_DEV float2 get(const T* p, float sc) { return lo(*p, sc); }
};

struct ImgArgs {
  const void* D;            // ring in the element form FMT of the kernel
  const float* scales;      // FMT 2: scale of each (chgroup, coarse DM, slot) row,
  const long long* sc_base; //   at scales[sc_base[g*n_coarse + c] + slot]
  const float* amax;        // FMT 0, 1: (amax_rows, G * n_coarse) bound of every |part|
                            //   stage 1 wrote for (chgroup, coarse DM) in a chunk of
                            //   amax_chunk stage-1 times, row (chunk mod amax_rows)
  const int* shift2;        // (G * n_coarse) stage-2 delays: ring time - stage-1 time
  int amax_chunk, amax_rows;
  const long long* seg_base;  // (G * n_coarse) ring segment of (chgroup, coarse DM)
  const int* seg_depth;       // (G * n_coarse) time slots of each segment
  int n_coarse;
  const unsigned* c_meta;   // (cell_base[G]) per pattern cell: tgt | conj << 16 | g << 17;
                            // 0xffffffff pads each chgroup's run to a multiple of 64
  const int* cell_base;     // (G + 1) multiples of 64
  const int2* c2;           // (n_c2) second targets: {cell | g << 16, tgt | conj << 16}
  int n_c2;
  const int* thr_b;         // (THREADS + 1) S range [thr_b[i], thr_b[i+1]) of thread i
  const uint4* gmeta;       // (MAXE / EPV, THREADS) 16 bytes per (chunk, thread): EPV
                            //   entries col | n' << NP_SH | q << Q_SH | last of its slot
                            //   << LAST_SH (the 32-bit form also packed | parity(u+w) << 1
                            //   at ROT_SH); ImgGeom gives the form of each N
  const unsigned long long* srot;  // 16-bit form: (THREADS) 2 bits per entry, packed |
                                   // parity(u+w) << 1; unused (may be null) at N = 512
  const int* dcols;         // (n_dense) packed columns that need the LC-point transform
  const unsigned long long* dmask;  // (n_dense) occupied slots n' of each
  int n_dense;
  const int* kcols;         // (n_const) col | has entries << 16: every entry at n' = 0
  int n_const;
  int n_s, s_stride;        // s_stride: even, >= n_s (the split S arrays in shared memory)
  int s_mult_log2;          // ceil(log2) of the most contributions to one S entry
  const int* d_pitch;       // (G) cells (row pitch) of each chgroup's segments
  const int* n_filled;      // (G) pattern cells of each chgroup
  const int* sfine;         // (n_fine, G)
  const int* f2c;           // (n_fine)
  const float2* tw;         // (N) W_N^e = exp(+2 pi i e / N)
  int f0, n_f, G;
  long long t0;
  int n_t;
  int fftshift;
  float* out;               // (n_f, n_t, N, N)
  int* status;
};

constexpr int IMG_MAX_G = 64;
#ifndef IMG_COMBINE_U
#define IMG_COMBINE_U 8   // 64-entry double chunks per warp in flight in the combine
#endif

// Geometry of image_kernel<N>.
//  * Column pass: N = FOLD * LC output rows in FOLD passes of LC rows; an
//    LC-point column transform is two C1-point steps (LC = C1 * C1).
//  * Row transforms: N = R1 * R2 on a group of R1 threads, each holding R2
//    points (an R2-point step, a transpose, R2 / R1 R1-point steps).
//  * N = 512: FOLD 8 (64-row passes), 512 threads, one CTA per SM with all
//    512 TMEM columns, 32-bit entry metadata (8 bits of column); the combine's
//    S arrays (int32 real and imaginary parts) take 192 KB of shared memory.
//  * N = 64, 256: FOLD 4, 256 threads, three CTAs per SM with 128 TMEM
//    columns each, 16-bit entry metadata.
// TMEM: warps w, w + 4, w + 8, ... reach the same 32 lanes; each takes an
// equal share of the CTA's columns, two 32-bit columns per complex S entry.
template <int N>
struct ImgGeom {
  static constexpr int FOLD = (N == 512) ? 8 : 4;
  static constexpr int LC = N / FOLD;             // folded column length
  static constexpr int C1 = (LC == 64) ? 8 : 4;    // LC = C1 * C1
  static constexpr int NC = N / 2;                // packed columns
  static constexpr int P = NC + 2;                // buffer row pitch (float2), = 2 mod 16
  static constexpr int R1 = (N == 64) ? 8 : 16;   // threads per row transform
  static constexpr int R2 = N / R1;               // points per thread
  static constexpr int THREADS = (N == 512) ? 512 : 256;
  static constexpr int CTAS = (N == 512) ? 1 : 3; // resident CTAs per SM
  static constexpr int TMEM_COLS = (N == 512) ? 512 : 128;
  static constexpr int WARP_COLS = TMEM_COLS / (THREADS / 128);  // columns per warp
  static constexpr int MAXE = WARP_COLS / 2;      // S entries per thread
  static constexpr bool META32 = (N == 512);
  // entry metadata fields: column | n' << NP_SH | q << Q_SH | last << LAST_SH
  // (32-bit form also: packed << ROT_SH | parity(u + w) << ROT_SH + 1)
  static constexpr int NP_SH = META32 ? 8 : 7;
  static constexpr int Q_SH = META32 ? 14 : 13;
  static constexpr int LAST_SH = META32 ? 17 : 15;
  static constexpr int ROT_SH = 18;
  static constexpr int CG = THREADS / C1;         // column groups
  static constexpr int RG = THREADS / R1;         // row groups
  static constexpr int BUF = LC * P;              // float2 slots of the column buffer
  // S entries the combine's split int32 arrays hold
  static constexpr int SCAP = (N == 512) ? 24576 : BUF;
  static constexpr size_t BUFB = (size_t)(BUF > SCAP ? BUF : SCAP) * 8;
  // 32-bit form: the fold reads compact tables that follow gmeta in its
  // buffer (a nibble q | last << 3 per entry, [chunk][thread]; the first slot
  // of each thread; the slots' column-buffer offsets n' P + w' as uint16),
  // copied per image into the part of buf the column buffer leaves free
  static constexpr int MAXC = MAXE / 8;                         // 8-entry chunks
  static constexpr size_t GM_BYTES = (size_t)(MAXE / 4) * THREADS * 16;
  static constexpr size_t FC_BYTES = (size_t)MAXC * THREADS * 4;
  static constexpr size_t TS_BYTES = (size_t)((THREADS + 1 + 3) / 4) * 16;
  static constexpr size_t ROT_BYTES = (size_t)THREADS * 16;  // 2 bits x 64 entries
  static constexpr int MAX_SLOTS = LC * NC;
  static_assert(C1 * C1 == LC && R1 * R2 == N && R2 % R1 == 0, "unsupported size");
  static_assert(2 * P >= N, "a row pair's slots must hold the transpose and two output rows");
  static_assert((2 * P * 8) % 16 == 0, "row-pair regions must stay 16-byte aligned");
  static_assert(META32 ? (NC <= 256 && LC <= 64 && FOLD <= 8)
                       : (NC <= 128 && LC <= 64 && FOLD <= 4),
                "entry metadata field widths");
  static_assert(MAXE % 8 == 0 && MAXE <= 64, "whole 8-entry chunks, 64-bit rotation masks");
  static_assert(LC <= 64, "one 64-bit occupancy mask per column");
  // buf | tw (N) | rtw (R1*R2) | ctw (C1*C1) | slice pointers | cell bases |
  // ends of the chgroups' cells | slice scales | TMEM address | k
  static constexpr size_t SMEM = BUFB + (size_t)(N + R1 * R2 + C1 * C1) * 8 + IMG_MAX_G * 8 +
                                 (IMG_MAX_G + 1) * 4 + IMG_MAX_G * 4 + IMG_MAX_G * 4 + 16;
  static_assert(SMEM <= 227 * 1024, "shared memory of one CTA");
  static_assert(!META32 || (size_t)BUF * 8 + FC_BYTES + (size_t)MAX_SLOTS * 2 <= BUFB,
                "the fold's tables fit beside the column buffer");
  static_assert(GM_BYTES % 16 == 0 && FC_BYTES % 16 == 0 && TS_BYTES % 16 == 0 &&
                    ROT_BYTES % 16 == 0,
                "every table after gmeta starts 16-byte aligned");
  static_assert(!META32 || ROT_SH == LAST_SH + 1,
                "the 32-bit entry's rotation bits follow its last bit");
};

// The 8 metadata entries of chunk c of this thread (entries 8c .. 8c + 7).
template <int N>
DSB_DEV void load_meta8(const uint4* gm, int c, int tid, unsigned (&m)[8]) {
  using Gm = ImgGeom<N>;
  if constexpr (Gm::META32) {
    const uint4 a = __ldg(gm + (2 * c) * Gm::THREADS + tid);
    const uint4 b = __ldg(gm + (2 * c + 1) * Gm::THREADS + tid);
    m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
    m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
  } else {
    const uint4 a = __ldg(gm + c * Gm::THREADS + tid);
    const unsigned w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
    for (int j = 0; j < 8; ++j) m[j] = (w[j >> 1] >> (16 * (j & 1))) & 0xffffu;
  }
}

template <int N, int FMT>
__global__ void __launch_bounds__(ImgGeom<N>::THREADS, ImgGeom<N>::CTAS)
    image_kernel(const ImgArgs A) {
  using Elem = typename RingElem<FMT>::T;
  using Gm = ImgGeom<N>;
  constexpr int FOLD = Gm::FOLD, LC = Gm::LC, C1 = Gm::C1, NC = Gm::NC, P = Gm::P,
                R1 = Gm::R1, R2 = Gm::R2, THREADS = Gm::THREADS, MAXE = Gm::MAXE;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  float2* buf = reinterpret_cast<float2*>(smem_raw);  // S in step 1, columns in 2-3
  float2* tw = reinterpret_cast<float2*>(smem_raw + Gm::BUFB);
  // twiddles laid out so that the lanes of a group read consecutive slots:
  // rtw[m2*R1 + j] = W_N^(j m2), ctw[m1*C1 + j] = W_LC^(j m1)
  float2* rtw = tw + N;
  float2* ctw = rtw + R1 * R2;
  const Elem** s_slice = reinterpret_cast<const Elem**>(ctw + C1 * C1);
  int* s_cbase = reinterpret_cast<int*>(s_slice + IMG_MAX_G);
  int* s_end = s_cbase + IMG_MAX_G + 1;
  float* s_scale = reinterpret_cast<float*>(s_end + IMG_MAX_G);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(s_scale + IMG_MAX_G);
  int* s_fixk = reinterpret_cast<int*>(s_tmem + 1);  // S holds S * 2^k as int32

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  for (int i = tid; i < N; i += THREADS) tw[i] = A.tw[i];
  for (int i = tid; i < R1 * R2; i += THREADS)
    rtw[i] = A.tw[((i % R1) * (i / R1)) & (N - 1)];
  for (int i = tid; i < C1 * C1; i += THREADS)
    ctw[i] = A.tw[((i % C1) * (i / C1) * (N / LC)) & (N - 1)];
  for (int g = tid; g <= A.G; g += THREADS) s_cbase[g] = A.cell_base[g];
  for (int g = tid; g < A.G; g += THREADS) s_end[g] = A.cell_base[g] + A.n_filled[g];
  // this thread's S entries [sb, sb + sn), whole slots
  const int sb = __ldg(A.thr_b + tid);
  const int sn = __ldg(A.thr_b + tid + 1) - sb;
  // 32-bit form: this thread's first slot and the number of slots (the
  // fold's compact tables after gmeta)
  int sl0 = 0, n_sl = 0;
  if constexpr (Gm::META32) {
    const int* ts = reinterpret_cast<const int*>(reinterpret_cast<const uint8_t*>(A.gmeta) +
                                                 Gm::GM_BYTES + Gm::FC_BYTES);
    sl0 = __ldg(ts + tid);
    n_sl = __ldg(ts + THREADS);
  }
  const bool bad_range = sn < 0 || sn > MAXE || sb < 0 || sb + sn > A.n_s ||
                         n_sl < 0 || n_sl > Gm::MAX_SLOTS || sl0 < 0 || sl0 > n_sl;
  bool bad_base = false;  // each chgroup's run: whole 64-entry pairs of chunks
  for (int g = tid; g <= A.G; g += THREADS) bad_base |= (A.cell_base[g] & 63) != 0;
  if (__syncthreads_or(bad_range || bad_base)) {
    if (tid == 0) dsb_flag(A.status, DSB_E_CAPACITY);
    return;  // every thread leaves, before any TMEM is taken
  }
  // rotation bits: 2 per entry (packed | parity << 1); the 16-bit form's in
  // srot, the 32-bit form's in the compact tables after gmeta (entry i at
  // bits 2 (i % 16) of word i / 16)
  const unsigned long long srot = Gm::META32 ? 0ull : __ldg(A.srot + tid);
  uint4 rot32 = make_uint4(0u, 0u, 0u, 0u);
  if constexpr (Gm::META32)
    rot32 = __ldg(reinterpret_cast<const uint4*>(reinterpret_cast<const uint8_t*>(A.gmeta) +
                                                 Gm::GM_BYTES + Gm::FC_BYTES + Gm::TS_BYTES) +
                  tid);
  const int nch = (__reduce_max_sync(0xffffffffu, sn) + 7) >> 3;  // 8-entry chunks, per warp
  if (warp == 0) {
    tmem_alloc(s_tmem, Gm::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *s_tmem + ((uint32_t)((warp & 3) * 32) << 16) +
                         (uint32_t)((warp >> 2) * Gm::WARP_COLS);

  const int n_tot = A.cell_base[A.G];
  // 0.5 / N^2 is a power of two, applied to S on its way into TMEM: scaling
  // every input of the transforms by a power of two scales every rounded
  // intermediate exactly, so the images are the bits the scale at the end
  // would give, without 2 N^2 multiplies per image
  const float scale = 0.5f / (float)(N * N);
  static_assert((N & (N - 1)) == 0, "0.5 / N^2 must be a power of two");
  const int n_img = A.n_f * A.n_t;
  // column groups: C1 lanes; row groups: R1 lanes (groups never straddle warps)
  const int cgi = tid / C1, cj = tid % C1;
  const unsigned cmask = ((1u << C1) - 1u) << (lane / C1 * C1);
  const int rgi = tid / R1, rj = tid % R1;
  const unsigned rmask = ((1u << R1) - 1u) << (lane / R1 * R1);
  const int shift_rot = A.fftshift ? 2 : 0;
  const uint4* gmeta = A.gmeta;

  for (int img = blockIdx.x; img < n_img; img += gridDim.x) {
    // fine DM fastest: CTAs that run together share coarse-DM slices in L2
    const int fl = img % A.n_f, t = img / A.n_f;
    const int f = A.f0 + fl;
    const int c = A.f2c[f];
    const long long ta = A.t0 + t;
    // (the previous image is done with buf and s_slice: its last pass ended
    // with a barrier, and the first image follows the one after the TMEM
    // allocation)
    if (warp == 0) {
      float smax = 0.f;
      for (int g = lane; g < A.G; g += 32) {
        const int gc = g * A.n_coarse + c;
        const long long dep = A.seg_depth[gc];
        long long slot = (ta - A.sfine[(long long)f * A.G + g]) % dep;
        if (slot < 0) slot += dep;
        s_slice[g] = static_cast<const Elem*>(A.D) + A.seg_base[gc] + slot * A.d_pitch[g];
        float sc = 1.f, bound;
        if constexpr (FMT == 2) {
          sc = A.scales[A.sc_base[gc] + slot];
          bound = sc;
        } else {
          // stage-1 time of the value read, its chunk's bound row
          const long long t1 = ta - A.sfine[(long long)f * A.G + g] - A.shift2[gc];
          const long long ch = t1 >= 0 ? t1 / A.amax_chunk
                                       : -((A.amax_chunk - 1 - t1) / A.amax_chunk);
          long long row = ch % A.amax_rows;
          if (row < 0) row += A.amax_rows;
          bound = A.amax[row * (long long)A.G * A.n_coarse + gc];
        }
        s_scale[g] = sc;
        smax = fmaxf(smax, bound);
      }
      // Fixed point, S summed as S * 2^k in int32.  Every part is at most
      // 128 x its row's scale (FMT 2) or its row's bound x (1 + 2^-8) (the
      // bf16 rounding; FMT 0, 1), so with 2^k = 2^(22 or 28 - ilogb(max) -
      // s_mult_log2) a part stays below 2^(30 - s_mult_log2) and any S
      // entry's sum below 2^30.
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
      const bool ok = smax >= 0.f && smax <= 3.0e38f;
      const int k = (ok && smax > 0.f)
                        ? min(100, (FMT == 2 ? 22 : 28) - ilogbf(smax) - A.s_mult_log2)
                        : 0;
      if (!ok && lane == 0) dsb_flag(A.status, DSB_E_ARG);
      for (int g = lane; g < A.G; g += 32) s_scale[g] = ldexpf(ok ? s_scale[g] : 0.f, k);
      if (lane == 0) *s_fixk = k;
    }
    {
      float4* b4 = reinterpret_cast<float4*>(buf);
      for (int i = tid; i < A.s_stride / 2; i += THREADS) b4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    // ---- 1. combine into S (shared-memory int32 atomics, fixed point) ----
    {
      // separate real and imaginary arrays: a warp's 32 atomics spread over
      // all 32 banks instead of the even (or odd) half
      float* s_re = reinterpret_cast<float*>(buf);
      float* s_im = s_re + A.s_stride;
      auto add = [&](unsigned m, float2 v) {
        const unsigned t = m & 0xffffu;
        if (!DSB_INB(t, A.s_stride, A.status)) return;
        // v is already scaled by 2^k: integer atomics (native, no
        // compare-and-swap loop) and a sum that does not depend on order
        const int re = __float2int_rn(v.x), im = __float2int_rn(v.y);
        atomicAdd(reinterpret_cast<int*>(s_re) + t, re);
        atomicAdd(reinterpret_cast<int*>(s_im) + t, ((m >> 16) & 1u) ? -im : im);
      };
      // warp w takes the 64-entry double chunks w, w + NW, ... of c_meta in
      // order, each lane two adjacent cells with one metadata and one ring
      // load; each chgroup's run is a whole number of double chunks, so the
      // chgroup, its first entry and its ring row stay in registers and
      // change only at a run boundary (warp-uniform), and the shared-memory
      // pipe is left to the atomics.  16 cells in flight per thread (8 was
      // 1.4 % slower over the whole kernel at the 256^2 workload).
      using Elem2 = typename RingElem<FMT>::T2;
      constexpr int U = IMG_COMBINE_U, NW = THREADS / 32;
      const int n_dch = n_tot >> 6;
      // forms 0 and 1: one factor 2^k for every chgroup
      const float fix = s_scale[0];
      const uint2* cm2 = reinterpret_cast<const uint2*>(A.c_meta);
      int g = -1, g_lo = 0, g_hi = 0, g_end = 0;
      float g_sc = 1.f;
      const Elem* src = static_cast<const Elem*>(A.D);
      for (int c0 = warp; c0 < n_dch; c0 += NW * U) {
        // raw ring words: decoded only in the add loop below, so that no
        // instruction waits on a load before the batch's other loads issue
        uint2 m[U];
        Elem2 v[U];
        float sc[U];
#pragma unroll
        for (int q = 0; q < U; ++q) {
          const int ch = c0 + NW * q;
          m[q] = make_uint2(0xffffffffu, 0xffffffffu);
          v[q] = RingElem<FMT>::zero2();
          sc[q] = 1.f;
          if (ch < n_dch) {
            while (64 * ch >= g_hi) {
              ++g;
              g_lo = s_cbase[g];
              g_hi = s_cbase[g + 1];
              g_end = s_end[g];
              src = s_slice[g];
              g_sc = s_scale[g];
            }
            // cells e, e + 1 (e even): both inside the row's pitch whenever
            // e is a pattern cell (the pitch is n_filled rounded up to 4)
            const int e = 64 * ch + 2 * lane;
            if (e < g_end && DSB_INB(e - g_lo + 1, A.d_pitch[g], A.status)) {
              m[q] = __ldg(cm2 + (e >> 1));
              v[q] = *reinterpret_cast<const Elem2*>(src + (e - g_lo));
              sc[q] = g_sc;
            }
          }
        }
#pragma unroll
        for (int q = 0; q < U; ++q) {
          const float f = FMT == 2 ? sc[q] : fix;
          if (m[q].x != 0xffffffffu) add(m[q].x, RingElem<FMT>::lo(v[q], f));
          if (m[q].y != 0xffffffffu) add(m[q].y, RingElem<FMT>::hi(v[q], f));
        }
      }
      for (int i = tid; i < A.n_c2; i += THREADS) {
        const int2 cm = __ldg(A.c2 + i);
        if (!DSB_INB(cm.x & 0xffff, A.d_pitch[(cm.x >> 16) & (IMG_MAX_G - 1)], A.status))
          continue;
        add((unsigned)cm.y,
            RingElem<FMT>::get(s_slice[(cm.x >> 16) & (IMG_MAX_G - 1)] + (cm.x & 0xffff),
                               s_scale[(cm.x >> 16) & (IMG_MAX_G - 1)]));
      }
    }
    __syncthreads();
    // ---- this thread's S entries into TMEM, with the rotation that does not
    //      depend on the pass (i for the packed column N/2, -1 for the
    //      fftshift checkerboard) already applied ----
    {
      const float* s_re = reinterpret_cast<const float*>(buf);
      const float* s_im = s_re + A.s_stride;
      const float unfix = ldexpf(scale, -*s_fixk);  // 2^-k x 0.5 / N^2
      for (int c = 0; c < nch; ++c) {
        // this chunk's 16 rotation bits (32-bit form)
        unsigned rw = 0u;
        if constexpr (Gm::META32) {
          const unsigned w2 = (c & 2) ? ((c & 4) ? rot32.w : rot32.y) : ((c & 4) ? rot32.z : rot32.x);
          rw = (c & 1) ? (w2 >> 16) : w2;
        }
        uint32_t r[16];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int i = 8 * c + j;
          float2 v = make_float2(0.f, 0.f);
          if (i < sn) {
            unsigned b;
            if constexpr (Gm::META32) b = (rw >> (2 * j)) & 3u;
            else b = (unsigned)(srot >> (2 * i)) & 3u;
            const float2 x = make_float2(__int2float_rn(__float_as_int(s_re[sb + i])) * unfix,
                                         __int2float_rn(__float_as_int(s_im[sb + i])) * unfix);
            v = crot_rt(x, (b & 1u) + ((b & 2u) ? (unsigned)shift_rot : 0u));
          }
          r[2 * j] = __float_as_uint(v.x);
          r[2 * j + 1] = __float_as_uint(v.y);
        }
        tmem_st16(tbase + 16 * c, r);
      }
      tmem_st_wait();
    }
    __syncthreads();  // S is read: buf is free for the passes
    if constexpr (Gm::META32) {
      // the fold's compact tables into the part of buf past the column buffer
      // (the combine's S arrays overlapped it): this thread's nibble words,
      // and every slot's offset (16-byte copies; slot_off is padded to 8)
      uint32_t* s_code = reinterpret_cast<uint32_t*>(buf + Gm::BUF);
      const uint8_t* gt = reinterpret_cast<const uint8_t*>(A.gmeta) + Gm::GM_BYTES;
      const uint32_t* g_code = reinterpret_cast<const uint32_t*>(gt);
      for (int c = 0; c < nch; ++c) s_code[c * THREADS + tid] = __ldg(g_code + c * THREADS + tid);
      const uint4* g_slot =
          reinterpret_cast<const uint4*>(gt + Gm::FC_BYTES + Gm::TS_BYTES + Gm::ROT_BYTES);
      uint4* s_slot4 = reinterpret_cast<uint4*>(s_code + Gm::MAXC * THREADS);
      for (int i = tid; i < (n_sl + 7) / 8; i += THREADS) s_slot4[i] = __ldg(g_slot + i);
      __syncthreads();
    }

    for (int p = 0; p < FOLD; ++p) {
      // ---- 2a. fold S into the occupied slots (n', col) of buf: each slot's
      //      entries are consecutive in one thread's range, written once
      //      after the last of them ----
      // (one copy of the loop per pass, so that the rotation W_FOLD^(q p)
      // needs as little work as the pass allows: none for p = 0, a sign for
      // p = FOLD/2, a swap and signs for the other even multiples, and one
      // multiply by W_8 for the odd ones)
      auto fold = [&](auto pass) {
        constexpr unsigned PP = decltype(pass)::value;
        float2 acc = make_float2(0.f, 0.f);
        if constexpr (Gm::META32) {
          // compact tables in shared memory: one nibble word per chunk, and
          // the offset of each of this thread's slots, in order
          const uint32_t* s_code = reinterpret_cast<const uint32_t*>(buf + Gm::BUF);
          const uint16_t* s_soff = reinterpret_cast<const uint16_t*>(s_code + Gm::MAXC * THREADS);
          int si = sl0;
          for (int c = 0; c < nch; ++c) {
            const uint32_t cw = s_code[c * THREADS + tid];
            uint32_t r[16];
            tmem_ld16_wait(tbase + 16 * c, r);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              if (8 * c + j < sn) {
                const unsigned code = (cw >> (4 * j)) & 15u;
                float2 v = make_float2(__uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 1]));
                if constexpr (PP != 0) {
                  // W_8^k = i^(k >> 1) x (W_8 if k is odd), k = q p mod 8
                  const unsigned k = ((code & 7u) * PP) & 7u;
                  if constexpr (PP & 1u) {
                    if (k & 1u) v = cmul_w8(v);
                  }
                  v = crot_rt(v, k >> 1);
                }
                acc = cadd(acc, v);
                if (code & 8u) {
                  if (DSB_INB(si, n_sl, A.status)) {
                    const unsigned off = s_soff[si];
                    if (DSB_INB(off, Gm::BUF, A.status)) buf[off] = acc;
                  }
                  ++si;
                  acc = make_float2(0.f, 0.f);
                }
              }
            }
          }
          return;
        }
        unsigned md_next[8];
        load_meta8<N>(gmeta, 0, tid, md_next);
        for (int c = 0; c < nch; ++c) {
          unsigned mw[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) mw[j] = md_next[j];
          // next chunk's metadata loads under this one's
          if (c + 1 < nch) load_meta8<N>(gmeta, c + 1, tid, md_next);
          uint32_t r[16];
          tmem_ld16_wait(tbase + 16 * c, r);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (8 * c + j < sn) {
              const unsigned m = mw[j];
              float2 v = make_float2(__uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 1]));
              const unsigned q = (m >> Gm::Q_SH) & (FOLD - 1);
              if constexpr (PP != 0) {
                if constexpr (FOLD == 4) {
                  if constexpr (PP == 2) {
                    const unsigned sgn = (q & 1u) << 31;  // i^(2q) = (-1)^q
                    v = make_float2(__uint_as_float(__float_as_uint(v.x) ^ sgn),
                                    __uint_as_float(__float_as_uint(v.y) ^ sgn));
                  } else {
                    v = crot_rt(v, q * PP);
                  }
                } else {
                  // W_8^k = i^(k >> 1) x (W_8 if k is odd), k = q p mod 8
                  const unsigned k = (q * PP) & 7u;
                  if constexpr (PP & 1u) {
                    if (k & 1u) v = cmul_w8(v);
                  }
                  v = crot_rt(v, k >> 1);
                }
              }
              acc = cadd(acc, v);
              if ((m >> Gm::LAST_SH) & 1u) {
                buf[((m >> Gm::NP_SH) & (LC - 1)) * P + (m & (NC - 1))] = acc;
                acc = make_float2(0.f, 0.f);
              }
            }
          }
        }
      };
      switch (p) {
        case 0: fold(std::integral_constant<unsigned, 0>{}); break;
        case 1: fold(std::integral_constant<unsigned, 1>{}); break;
        case 2: fold(std::integral_constant<unsigned, 2>{}); break;
        case 3: fold(std::integral_constant<unsigned, 3>{}); break;
        default:
          if constexpr (FOLD == 8) {
            switch (p) {
              case 4: fold(std::integral_constant<unsigned, 4>{}); break;
              case 5: fold(std::integral_constant<unsigned, 5>{}); break;
              case 6: fold(std::integral_constant<unsigned, 6>{}); break;
              default: fold(std::integral_constant<unsigned, 7>{}); break;
            }
          }
          break;
      }
      __syncthreads();
      // ---- 2b. column transforms of pass p (in place in buf); only the
      //      occupied slots of a column are read ----
      for (int di = cgi; di < A.n_dense; di += Gm::CG) {
        const int col = __ldg(A.dcols + di) & (NC - 1);
        const unsigned long long occ = __ldg(A.dmask + di);
        float2* colp = buf + col;
        float2 y[C1];
#pragma unroll
        for (int k = 0; k < C1; ++k) {
          const int n1 = cj + C1 * k;
          y[k] = ((occ >> n1) & 1ull) ? cmul(colp[n1 * P], tw[(n1 * p) & (N - 1)])
                                      : make_float2(0.f, 0.f);
        }
        idftR<C1>(y);
#pragma unroll
        for (int m1 = 1; m1 < C1; ++m1) y[m1] = cmul(y[m1], ctw[m1 * C1 + cj]);
        __syncwarp(cmask);  // every lane has read its slots of the column
#pragma unroll
        for (int m1 = 0; m1 < C1; ++m1) colp[((cj ^ m1) + C1 * m1) * P] = y[m1];
        __syncwarp(cmask);
#pragma unroll
        for (int jj = 0; jj < C1; ++jj) y[jj] = colp[((jj ^ cj) + C1 * cj) * P];
        __syncwarp(cmask);
        idftR<C1>(y);
#pragma unroll
        for (int m2 = 0; m2 < C1; ++m2) colp[(cj + C1 * m2) * P] = y[m2];
      }
      // constant columns: every row holds the folded slot n' = 0 (row 0
      // itself is already in place); columns without entries are zero.  The
      // lanes of a warp take consecutive columns of one row (no bank
      // conflicts), the warps take rows m = warp (mod warps).
      for (int k = lane; k < A.n_const; k += 32) {
        const int kc = __ldg(A.kcols + k);
        const int col = kc & (NC - 1);
        const bool has = kc >> 16;
        const float2 y0 = has ? buf[col] : make_float2(0.f, 0.f);
        for (int m = warp; m < LC; m += THREADS / 32)
          if (m || !has) buf[m * P + col] = y0;
      }
      __syncthreads();
      // ---- 3. row transforms: folded rows (2pr, 2pr + 1) are image rows
      //      FOLD*2pr + p and FOLD*(2pr+1) + p.  N = R1 * R2: thread rj holds
      //      points rj + R1 k2 (k2 < R2), takes their R2-point transform,
      //      twiddles it by W_N^(rj m2), and after the transpose owns the
      //      R1-point transforms of columns m2 = rj + R1 h, which give the
      //      outputs m2 + R2 m1 ----
      for (int pr = rgi; pr < LC / 2; pr += Gm::RG) {
        float2* reg = buf + 2 * pr * P;
        const float2* ra = reg;
        const float2* rb = reg + P;
        float2 a[R2];
#pragma unroll
        for (int k = 0; k < R2; ++k) {
          const int i = rj + R1 * k;
          float2 z;
          if (i == 0) {
            z = make_float2(ra[0].x, rb[0].x);
          } else if (i == N / 2) {
            z = make_float2(ra[0].y, rb[0].y);
          } else if (i < N / 2) {
            const float2 ya = ra[i], yb = rb[i];
            z = make_float2(ya.x - yb.y, ya.y + yb.x);   // ya + i yb
          } else {
            const float2 ya = ra[N - i], yb = rb[N - i];
            z = make_float2(ya.x + yb.y, -ya.y + yb.x);  // conj(ya) + i conj(yb)
          }
          a[k] = z;
        }
        idftR<R2>(a);
#pragma unroll
        for (int m2 = 1; m2 < R2; ++m2) a[m2] = cmul(a[m2], rtw[m2 * R1 + rj]);
        __syncwarp(rmask);  // every lane has read the pair's rows
#pragma unroll
        for (int m2 = 0; m2 < R2; ++m2) reg[m2 * R1 + (rj ^ (m2 & (R1 - 1)))] = a[m2];
        __syncwarp(rmask);
        constexpr int H = R2 / R1;
        float2 b[H][R1];
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int m2 = rj + R1 * h;
#pragma unroll
          for (int jj = 0; jj < R1; ++jj) b[h][jj] = reg[m2 * R1 + (jj ^ rj)];
        }
        const size_t ibase = ((size_t)fl * A.n_t + t) * N;
        float* ra_out = A.out + (ibase + FOLD * (2 * pr) + p) * N;
        float* rb_out = A.out + (ibase + FOLD * (2 * pr + 1) + p) * N;
        if constexpr (N == 512) {
          // outputs straight from registers: for each (h, m1) the group's
          // 16 lanes hold 16 consecutive pixels of each row (64 bytes), so
          // no staging through shared memory (whose pipe the transposes
          // already keep busy)
#pragma unroll
          for (int h = 0; h < H; ++h) {
            idftR<R1>(b[h]);
#pragma unroll
            for (int m1 = 0; m1 < R1; ++m1) {
              const int x = rj + R1 * h + R2 * m1;
              ra_out[x] = b[h][m1].x;
              rb_out[x] = b[h][m1].y;
            }
          }
        } else {
          __syncwarp(rmask);
          float* stage = reinterpret_cast<float*>(reg);
#pragma unroll
          for (int h = 0; h < H; ++h) {
            idftR<R1>(b[h]);
#pragma unroll
            for (int m1 = 0; m1 < R1; ++m1) {
              const int x = rj + R1 * h + R2 * m1;
              stage[x] = b[h][m1].x;
              stage[N + x] = b[h][m1].y;
            }
          }
          __syncwarp(rmask);
          float4* oa = reinterpret_cast<float4*>(ra_out);
          float4* ob = reinterpret_cast<float4*>(rb_out);
          const float4* s4 = reinterpret_cast<const float4*>(stage);
#pragma unroll
          for (int q = rj; q < N / 4; q += R1) {
            oa[q] = s4[q];
            ob[q] = s4[N / 4 + q];
          }
        }
      }
      __syncthreads();
    }
  }
  // every tcgen05.ld above was waited for; give the columns back
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(*s_tmem, Gm::TMEM_COLS);
  }
}

// Resident CTAs for image_kernel<N, FMT> on this device (the persistent grid).
// The occupancy API answers 1 CTA per SM for any kernel that allocates
// tensor memory (measured on B200 with CUDA 12.9), while the SM runs as many
// as its shared memory, registers and 512 TMEM columns hold (three at
// N <= 256, one at N = 512).  So the count is taken from those limits
// directly.
template <int N, int FMT>
int image_grid(int* blocks) {
  using Gm = ImgGeom<N>;
  static int cached = 0;
  if (!cached) {
    if (cudaFuncSetAttribute(image_kernel<N, FMT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Gm::SMEM) != cudaSuccess)
      return DSB_E_CUDA;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, image_kernel<N, FMT>) != cudaSuccess) return DSB_E_CUDA;
    int dev = 0, sms = 148, smem_sm = 0, smem_rsv = 0, regs_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    const int by_smem = smem_sm / ((int)Gm::SMEM + fa.sharedSizeBytes + smem_rsv);
    const int regs_cta = (fa.numRegs + 7) / 8 * 8 * Gm::THREADS;
    const int by_regs = regs_cta > 0 ? regs_sm / regs_cta : 1;
    const int occ = std::min({Gm::CTAS, by_smem, by_regs, 512 / Gm::TMEM_COLS});
    cached = std::max(1, occ) * sms;
  }
  *blocks = cached;
  return DSB_OK;
}

template <int N, int FMT>
int launch_image(const ImgArgs& A, int max_blocks, cudaStream_t stream) {
  using Gm = ImgGeom<N>;
  if (A.s_stride > Gm::SCAP) return DSB_E_CAPACITY;
  if (!Gm::META32 && !A.srot) return DSB_E_ARG;
  int blocks = 0;
  const int rc = image_grid<N, FMT>(&blocks);
  if (rc != DSB_OK) return rc;
  if (max_blocks > 0) blocks = std::min(blocks, max_blocks);
  blocks = std::max(1, std::min(blocks, A.n_f * A.n_t));
  image_kernel<N, FMT><<<blocks, Gm::THREADS, Gm::SMEM, stream>>>(A);
  return launch_status();
}

// ===========================================================================
// Dense inverse real 2-D FFT of Hermitian half spectra, the transform of
// torch.fft.irfft2(half, s=(N, N)) (norm "backward"): half [n_img][N][N/2+1]
// complex64 -> out [n_img][N][N] float32.  Used where the combine is dense
// (GpuImager.process_cube, image/imager_gpu.py:575-605).  Two passes:
//  1. columns: an N-point inverse complex transform over u of every column
//     w in place in half (CTA = 16 adjacent columns of one image, staged in
//     shared memory with a pitch of 17 so that a column's slots fall in
//     different banks);
//  2. rows: two rows per complex transform (x_a + i x_b) as in the image
//     kernel; the imaginary parts of columns 0 and N/2 are dropped (a
//     Hermitian spectrum makes them zero; numpy and cuFFT drop them too).
// Both passes use the R1 x R2 factorisation of the image kernel.
// ===========================================================================
constexpr int FFT_CW = 16;  // columns per CTA of the column pass

template <int N>
struct DenseGeom {
  static constexpr int R1 = (N <= 32) ? 4 : (N <= 128 ? 8 : 16);
  static constexpr int R2 = N / R1;
  static constexpr int NH = N / 2 + 1;
  static constexpr int CP = FFT_CW + 1;         // pitch of the staged columns (float2)
  static constexpr int COL_THREADS = FFT_CW * R1;
  static constexpr int ROW_GROUPS = 8;          // row pairs per CTA of the row pass
  static constexpr int ROW_THREADS = ROW_GROUPS * R1;
  static_assert(R1 * R2 == N && R2 % R1 == 0, "unsupported size");
};

// One N-point inverse transform by a group of R1 threads (thread rj) over
// the N values at slots p(i) of shared memory, in place, natural order out.
template <int N, typename Slot>
DSB_DEV void group_idft(Slot p, int rj, unsigned mask, const float2* rtw) {
  using Dg = DenseGeom<N>;
  constexpr int R1 = Dg::R1, R2 = Dg::R2, H = R2 / R1;
  float2 a[R2];
#pragma unroll
  for (int k = 0; k < R2; ++k) a[k] = *p(rj + R1 * k);
  idftR<R2>(a);
#pragma unroll
  for (int m2 = 1; m2 < R2; ++m2) a[m2] = cmul(a[m2], rtw[m2 * R1 + rj]);
  __syncwarp(mask);
#pragma unroll
  for (int m2 = 0; m2 < R2; ++m2) *p(m2 * R1 + (rj ^ (m2 & (R1 - 1)))) = a[m2];
  __syncwarp(mask);
  float2 b[H][R1];
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const int m2 = rj + R1 * h;
#pragma unroll
    for (int jj = 0; jj < R1; ++jj) b[h][jj] = *p(m2 * R1 + (jj ^ rj));
  }
  __syncwarp(mask);
#pragma unroll
  for (int h = 0; h < H; ++h) {
    idftR<R1>(b[h]);
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) *p(rj + R1 * h + R2 * m1) = b[h][m1];
  }
  __syncwarp(mask);
}

template <int N>
__global__ void __launch_bounds__(DenseGeom<N>::COL_THREADS)
    irfft2_cols_kernel(float2* __restrict__ half, const float2* __restrict__ twn) {
  using Dg = DenseGeom<N>;
  constexpr int R1 = Dg::R1, NH = Dg::NH, CP = Dg::CP;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  float2* col = reinterpret_cast<float2*>(smem_raw);   // [N][CP]
  float2* rtw = col + N * CP;                          // [R2][R1]
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < N; i += blockDim.x) rtw[i] = twn[((i % R1) * (i / R1)) & (N - 1)];
  const int w0 = blockIdx.x * FFT_CW;
  const int nw = min(FFT_CW, NH - w0);
  float2* img = half + (size_t)blockIdx.y * N * NH;
  for (int i = tid; i < N * FFT_CW; i += blockDim.x) {
    const int r = i / FFT_CW, c = i % FFT_CW;
    col[r * CP + c] = c < nw ? img[(size_t)r * NH + w0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int c = tid / R1, rj = tid % R1;
  const unsigned mask = ((1u << R1) - 1u) << (lane / R1 * R1);
  group_idft<N>([&](int i) { return col + i * CP + c; }, rj, mask, rtw);
  __syncthreads();
  for (int i = tid; i < N * FFT_CW; i += blockDim.x) {
    const int r = i / FFT_CW, cc = i % FFT_CW;
    if (cc < nw) img[(size_t)r * NH + w0 + cc] = col[r * CP + cc];
  }
}

template <int N>
__global__ void __launch_bounds__(DenseGeom<N>::ROW_THREADS)
    irfft2_rows_kernel(const float2* __restrict__ half, const float2* __restrict__ twn,
                       float* __restrict__ out) {
  using Dg = DenseGeom<N>;
  constexpr int R1 = Dg::R1, NH = Dg::NH;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  float2* rtw = reinterpret_cast<float2*>(smem_raw);   // [R2][R1]
  float2* reg0 = rtw + N;                              // [ROW_GROUPS][N]
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < N; i += blockDim.x) rtw[i] = twn[((i % R1) * (i / R1)) & (N - 1)];
  __syncthreads();
  const int grp = tid / R1, rj = tid % R1;
  const unsigned mask = ((1u << R1) - 1u) << (lane / R1 * R1);
  const int pr = blockIdx.x * Dg::ROW_GROUPS + grp;   // row pair (whole groups leave)
  if (pr >= N / 2) return;
  const float2* src = half + (size_t)blockIdx.y * N * NH;
  const float2* ra = src + (size_t)(2 * pr) * NH;
  const float2* rb = ra + NH;
  float2* reg = reg0 + grp * N;
  for (int i = rj; i < N; i += R1) {
    float2 z;
    if (i == 0) {
      z = make_float2(ra[0].x, rb[0].x);
    } else if (i == N / 2) {
      z = make_float2(ra[N / 2].x, rb[N / 2].x);
    } else if (i < N / 2) {
      const float2 ya = ra[i], yb = rb[i];
      z = make_float2(ya.x - yb.y, ya.y + yb.x);     // ya + i yb
    } else {
      const float2 ya = ra[N - i], yb = rb[N - i];
      z = make_float2(ya.x + yb.y, -ya.y + yb.x);    // conj(ya) + i conj(yb)
    }
    reg[i] = z;
  }
  __syncwarp(mask);
  group_idft<N>([&](int i) { return reg + i; }, rj, mask, rtw);
  // 1/N^2 (a power of two: exact)
  constexpr float scale = 1.0f / (float)(N * N);
  float* oa = out + ((size_t)blockIdx.y * N + 2 * pr) * N;
  float* ob = oa + N;
  for (int i = rj; i < N; i += R1) {
    const float2 v = reg[i];
    oa[i] = v.x * scale;
    ob[i] = v.y * scale;
  }
}

template <int N>
int launch_irfft2(float2* half, int n_img, const float2* twn, float* out, cudaStream_t stream) {
  using Dg = DenseGeom<N>;
  const size_t smem_c = (size_t)(N * Dg::CP + N) * sizeof(float2);
  const size_t smem_r = (size_t)(N + Dg::ROW_GROUPS * N) * sizeof(float2);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(irfft2_cols_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_c) != cudaSuccess ||
        cudaFuncSetAttribute(irfft2_rows_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_r) != cudaSuccess)
      return DSB_E_CUDA;
    attr = true;
  }
  const dim3 gc((Dg::NH + FFT_CW - 1) / FFT_CW, n_img);
  irfft2_cols_kernel<N><<<gc, Dg::COL_THREADS, smem_c, stream>>>(half, twn);
  const dim3 gr((N / 2 + Dg::ROW_GROUPS - 1) / Dg::ROW_GROUPS, n_img);
  irfft2_rows_kernel<N><<<gr, Dg::ROW_THREADS, smem_r, stream>>>(half, twn, out);
  return launch_status();
}

template <int N>
int image_geometry(int* g) {
  using Gm = ImgGeom<N>;
  g[0] = Gm::FOLD;
  g[1] = Gm::THREADS;
  g[2] = Gm::MAXE;
  g[3] = Gm::META32 ? 32 : 16;
  g[4] = Gm::SCAP;
  return DSB_OK;
}

}  // namespace

extern "C" {

int dsb_image_geometry(int n_grid, int* geom) {
  if (!geom) return DSB_E_ARG;
  switch (n_grid) {
    case 64: return image_geometry<64>(geom);
    case 256: return image_geometry<256>(geom);
    case 512: return image_geometry<512>(geom);
    default: return DSB_E_UNSUPPORTED;
  }
}

int dsb_irfft2(void* half, int n_img, int N, const void* twiddles, float* out,
               cudaStream_t stream) {
  if (!half || !twiddles || !out || n_img <= 0 || n_img > 65535) return DSB_E_ARG;
  if ((reinterpret_cast<uintptr_t>(half) & 7) || (reinterpret_cast<uintptr_t>(out) & 3))
    return DSB_E_ARG;
  float2* h = static_cast<float2*>(half);
  const float2* tw = static_cast<const float2*>(twiddles);
  switch (N) {
    case 32: return launch_irfft2<32>(h, n_img, tw, out, stream);
    case 64: return launch_irfft2<64>(h, n_img, tw, out, stream);
    case 128: return launch_irfft2<128>(h, n_img, tw, out, stream);
    case 256: return launch_irfft2<256>(h, n_img, tw, out, stream);
    case 512: return launch_irfft2<512>(h, n_img, tw, out, stream);
    default: return DSB_E_UNSUPPORTED;
  }
}

int dsb_image_fft(const void* D, int d_format, const long long* seg_base, const int* seg_depth,
                  const float* scales, const long long* sc_base, const float* amax,
                  const int* shift2, int amax_chunk, int amax_rows, int n_coarse,
                  const unsigned* c_meta, const int* cell_base, const void* c2, int n_c2,
                  const int* thr_b, const void* gmeta, const unsigned long long* srot, int n_s,
                  int s_mult, const int* dcols, const unsigned long long* dmask, int n_dense,
                  const int* kcols, int n_const, const int* d_pitch, const int* n_filled,
                  const int* sfine, const int* f2c, const void* twiddles, int f0, int n_f, int G,
                  int N, long long t0, int n_t, int fftshift, void* out, int max_blocks,
                  int* status, cudaStream_t stream) {
  if (!D || !seg_base || !seg_depth || n_coarse <= 0 || !c_meta || !cell_base ||
      (n_c2 > 0 && !c2) || n_c2 < 0 || !thr_b || !gmeta || n_s <= 0 ||
      n_s > 65536 || n_dense < 0 || n_const < 0 || (n_dense > 0 && (!dcols || !dmask)) ||
      (n_const > 0 && !kcols) || !d_pitch || !n_filled || !sfine || !f2c || !twiddles ||
      !out || !status || n_f <= 0 || n_t <= 0 || G <= 0 || G > IMG_MAX_G ||
      d_format < 0 || d_format > 2 || (d_format == 2 && (!scales || !sc_base)) ||
      (d_format != 2 && (!amax || !shift2 || amax_chunk <= 0 || amax_rows <= 0)) ||
      s_mult < 1 || s_mult > (1 << 20))
    return DSB_E_ARG;
  // two adjacent cells per load: 4-byte aligned cint8 pairs
  if (d_format == 2 && (reinterpret_cast<uintptr_t>(D) & 3)) return DSB_E_ARG;
  if ((reinterpret_cast<uintptr_t>(gmeta) & 15) || (reinterpret_cast<uintptr_t>(out) & 15))
    return DSB_E_ARG;
  if (n_dense + n_const != N / 2) return DSB_E_ARG;  // every packed column, once
  const int stride = (n_s + 1) & ~1;
  int mult_log2 = 0;
  while ((1 << mult_log2) < s_mult) ++mult_log2;
  ImgArgs A{D, scales, sc_base, amax, shift2, amax_chunk, amax_rows, seg_base, seg_depth, n_coarse, c_meta, cell_base, (const int2*)c2,
            n_c2, thr_b, (const uint4*)gmeta, srot, dcols, dmask, n_dense, kcols, n_const,
            n_s, stride, mult_log2, d_pitch, n_filled, sfine, f2c, (const float2*)twiddles, f0, n_f, G,
            t0, n_t, fftshift, (float*)out, status};
  switch (N) {
    case 64:
      return d_format == 2   ? launch_image<64, 2>(A, max_blocks, stream)
             : d_format == 1 ? launch_image<64, 1>(A, max_blocks, stream)
                             : launch_image<64, 0>(A, max_blocks, stream);
    case 256:
      return d_format == 2   ? launch_image<256, 2>(A, max_blocks, stream)
             : d_format == 1 ? launch_image<256, 1>(A, max_blocks, stream)
                             : launch_image<256, 0>(A, max_blocks, stream);
    case 512:
      return d_format == 2   ? launch_image<512, 2>(A, max_blocks, stream)
             : d_format == 1 ? launch_image<512, 1>(A, max_blocks, stream)
                             : launch_image<512, 0>(A, max_blocks, stream);
    default: return DSB_E_UNSUPPORTED;
  }
}

}  // extern "C"
