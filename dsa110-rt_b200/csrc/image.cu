// Fused fine-DM combine + 2-D inverse real FFT (sm_100a).
//
// One image per (fine DM f, time t):
//   G_h[u, w] = 0.5 * sum_e s_e(D[t - sf[f, g_e]][row_e]) * (-1)^(u+w),  w in [0, N/2]
//   img[x, y] = irfft2(G_h)[x, y]        (1/N^2 normalisation, numpy/torch "backward")
// which replaces fused_dequant_combine_per_fdm_half + torch.fft.irfft2
// (src/dsart/image/fused_combine_cuda.py:560-620, image/imager_gpu.py:590).
//
// Layout of the work: a cluster of CL CTAs owns one image at a time.  CTA r
// holds the half-spectrum columns [r*CW, ...) in shared memory (column-major,
// column stride N+1 to keep row reads conflict-free), combines them straight
// from the time-major stage-2 ring, runs the column transforms, and after a
// cluster barrier transforms its rows, reading the other CTAs' columns
// through distributed shared memory.  Two real output rows are packed into
// one complex transform (x_a + i x_b).
//
// Every N-point transform (N = R*R) runs on a group of R threads: an R-point
// DFT in registers, the twiddles w_N^(j*x1), one padded shared-memory
// transpose, and a second R-point DFT (the classic two-step factorisation).
#include "dsb_common.cuh"

#include <cooperative_groups.h>

#include <algorithm>

namespace cg = cooperative_groups;

namespace {

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

DSB_DEV float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
DSB_DEV float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
DSB_DEV float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
DSB_DEV float2 cmul_i(float2 a) { return make_float2(-a.y, a.x); }  // i * a

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

template <int R>
DSB_DEV void idftR(float2 (&a)[R]) {
  if constexpr (R == 16) idft16(a);
  else idft8(a);
}

// One N-point inverse complex transform (N = R*R) by the R threads of a group
// (thread j).  load(i) returns input element i; store(i, v) writes output i.
template <int R, typename Load, typename Store>
DSB_DEV void fft_group(int j, unsigned mask, float2* scr, const float2* tw, Load load,
                       Store store) {
  constexpr int N = R * R;
  float2 a[R];
#pragma unroll
  for (int k = 0; k < R; ++k) a[k] = load(j + R * k);
  idftR<R>(a);
#pragma unroll
  for (int x1 = 1; x1 < R; ++x1) a[x1] = cmul(a[x1], tw[(j * x1) & (N - 1)]);
#pragma unroll
  for (int x1 = 0; x1 < R; ++x1) scr[x1 * (R + 1) + j] = a[x1];
  __syncwarp(mask);
#pragma unroll
  for (int jj = 0; jj < R; ++jj) a[jj] = scr[j * (R + 1) + jj];
  __syncwarp(mask);
  idftR<R>(a);
#pragma unroll
  for (int x2 = 0; x2 < R; ++x2) store(j + R * x2, a[x2]);
}

struct ImgArgs {
  const float2* D;
  long long d_rows, d_mask;
  const int* sc_off;    // (CL + 1): rank r's scatter entries are [sc_off[r], sc_off[r+1])
  const int2* sc_meta;  // {cell | g << 16 | mirror << 31, target wl*(N+1) + u}
  const int* d_base;    // (G)
  const int* n_filled;  // (G)
  const int* sfine;     // (n_fine, G)
  const int* f2c;       // (n_fine)
  const float2* tw;     // (N) w_N^e = exp(+2 pi i e / N)
  int f0, n_f, G;
  long long t0;
  int n_t;
  int fftshift;
  float* out;           // (n_f, n_t, N, N)
  int* status;
};

template <int N, int CL>
struct ImgGeom {
  static constexpr int R = (N == 256) ? 16 : 8;
  static constexpr int NH = N / 2 + 1;
  static constexpr int CW = (NH + CL - 1) / CL;  // columns per CTA (last may have fewer)
  static constexpr int CS = N + 1;               // column stride (float2)
  static constexpr int HREG = (CW * CS + 1) / 2 * 2;  // H region, float2, 16-byte multiple
  static constexpr int RW = N / CL;              // output rows per CTA
  static constexpr int THREADS = 256;
  static constexpr int GROUPS = THREADS / R;
  static_assert((R * (R + 1) * 8) % 16 == 0, "group scratch must keep 16-byte alignment");
  static_assert(2 * N * 4 <= R * (R + 1) * 8, "two output rows must fit a group's scratch");
  static constexpr size_t SMEM = (size_t)HREG * 8 + (size_t)GROUPS * R * (R + 1) * 8 +
                                 (size_t)N * 8 + 48 * 8 + 48 * 4 + 256;
};

template <int N, int CL>
__global__ void __launch_bounds__(256, 1) image_kernel(const ImgArgs A) {
  using Gm = ImgGeom<N, CL>;
  constexpr int R = Gm::R, CW = Gm::CW, CS = Gm::CS, RW = Gm::RW, NH = Gm::NH;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  float2* H = reinterpret_cast<float2*>(smem_raw);
  float2* scr_all = H + Gm::HREG;  // 16-byte aligned (float4 staging)
  float2* tw = scr_all + Gm::GROUPS * R * (R + 1);
  const float2** s_slice = reinterpret_cast<const float2**>(tw + N);  // (G) slice starts
  int* s_misc = reinterpret_cast<int*>(s_slice + 48);                 // (G) n_filled

  int rank = 0;
  if constexpr (CL > 1) rank = (int)cg::this_cluster().block_rank();
  const int cluster_id = (int)blockIdx.x / CL;
  const int n_clusters = (int)gridDim.x / CL;
  const int tid = threadIdx.x, grp = tid / R, j = tid % R;
  float2* scr = scr_all + grp * R * (R + 1);
  // lanes of this thread's group inside its warp (groups never straddle warps)
  const unsigned gmask = (R == 32 ? 0xffffffffu : ((1u << R) - 1u)) << ((tid & 31) / R * R);
  const int w0 = rank * CW;
  const int ncol = min(CW, NH - w0);
  const int* sc_off = A.sc_off + rank;
  // base pointers of every rank's column block (own block is local)
  const float2* colbase[CL];
#pragma unroll
  for (int r = 0; r < CL; ++r) {
    colbase[r] = H;
    if constexpr (CL > 1) {
      if (r != rank) colbase[r] = cg::this_cluster().map_shared_rank(H, r);
    }
  }

  for (int i = tid; i < N; i += Gm::THREADS) tw[i] = A.tw[i];
  for (int g = tid; g < A.G; g += Gm::THREADS) s_misc[g] = A.n_filled[g];
  __syncthreads();

  const float scale = 1.0f / (float)(N * N);
  const int n_img = A.n_f * A.n_t;
  for (int img = cluster_id; img < n_img; img += n_clusters) {
    const int fl = img / A.n_t, t = img % A.n_t;
    const int f = A.f0 + fl;
    const int c = A.f2c[f];
    const long long ta = A.t0 + t;
    // per-image start of each chgroup's coarse-DM slice in the stage-2 ring
    for (int g = tid; g < A.G; g += Gm::THREADS)
      s_slice[g] = A.D + ((ta - A.sfine[(long long)f * A.G + g]) & A.d_mask) * A.d_rows +
                   A.d_base[g] + (long long)c * s_misc[g];
    for (int i = tid; i < CW * CS; i += Gm::THREADS) H[i] = make_float2(0.f, 0.f);
    __syncthreads();
    // ---- phase A: scatter every chgroup's stage-2 slice into my half-spectrum
    //      columns (shared-memory float atomics; entry = {cell | g<<16 |
    //      mirror<<31, target}) ----
    {
      const int e0 = sc_off[0], e1 = sc_off[1];
      constexpr int U = 4;
      int e = e0 + tid;
      for (; e + (U - 1) * Gm::THREADS < e1; e += U * Gm::THREADS) {
        int2 md[U];
        float2 x[U];
#pragma unroll
        for (int q = 0; q < U; ++q) md[q] = A.sc_meta[e + q * Gm::THREADS];
#pragma unroll
        for (int q = 0; q < U; ++q) x[q] = s_slice[(md[q].x >> 16) & 0x7fff][md[q].x & 0xffff];
#pragma unroll
        for (int q = 0; q < U; ++q) {
          atomicAdd(&H[md[q].y].x, x[q].x);
          atomicAdd(&H[md[q].y].y, md[q].x < 0 ? -x[q].y : x[q].y);
        }
      }
      for (; e < e1; e += Gm::THREADS) {
        const int2 md = A.sc_meta[e];
        const float2 x = s_slice[(md.x >> 16) & 0x7fff][md.x & 0xffff];
        atomicAdd(&H[md.y].x, x.x);
        atomicAdd(&H[md.y].y, md.x < 0 ? -x.y : x.y);
      }
    }
    __syncthreads();
    // ---- phase B: column transforms (along u) in place; the combine's 0.5
    //      and the fftshift checkerboard (-1)^(u+w) are applied on load ----
    for (int col = grp; col < ncol; col += Gm::GROUPS) {
      float2* colp = H + col * CS;
      const int w = w0 + col;
      fft_group<R>(j, gmask, scr, tw,
                   [&](int i) {
                     const float2 v = colp[i];
                     const float s = (A.fftshift && ((i + w) & 1)) ? -0.5f : 0.5f;
                     return make_float2(v.x * s, v.y * s);
                   },
                   [&](int i, float2 v) { colp[i] = v; });
    }
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();
    // ---- phase C: row transforms, two real rows per complex transform ----
    // Z[w] = Y_a[w] + i Y_b[w] (w <= N/2), conj-extended above N/2, with the
    // imaginary parts of Y[0] and Y[N/2] dropped (c2r convention).
    for (int pr = grp; pr < RW / 2; pr += Gm::GROUPS) {
      const int xa = rank * RW + 2 * pr, xb = xa + 1;
      auto colptr = [&](int w) -> const float2* {
        const int owner = w / CW;
        return colbase[owner] + (w - owner * CW) * CS;
      };
      auto load = [&](int i) -> float2 {
        if (i == 0 || i == N / 2) {
          const float2* cp = colptr(i);
          return make_float2(cp[xa].x, cp[xb].x);
        }
        if (i < N / 2) {
          const float2* cp = colptr(i);
          const float2 ya = cp[xa], yb = cp[xb];
          return make_float2(ya.x - yb.y, ya.y + yb.x);           // ya + i yb
        }
        const float2* cp = colptr(N - i);
        const float2 ya = cp[xa], yb = cp[xb];
        return make_float2(ya.x + yb.y, -ya.y + yb.x);            // conj(ya) + i conj(yb)
      };
      // rows x_a = Re, x_b = Im of the transform; staged through the group's
      // scratch and written as float4
      float* stage = reinterpret_cast<float*>(scr);
      fft_group<R>(j, gmask, scr, tw, load, [&](int i, float2 v) {
        stage[i] = v.x * scale;
        stage[N + i] = v.y * scale;
      });
      __syncwarp(gmask);
      float4* o4 = reinterpret_cast<float4*>(A.out + (((size_t)fl * A.n_t + t) * N + xa) * N);
      const float4* s4 = reinterpret_cast<const float4*>(stage);
#pragma unroll
      for (int q = j; q < N / 2; q += R) o4[q] = s4[q];
      __syncwarp(gmask);
    }
    // the other CTAs may still read my columns
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();
  }
}

template <int N, int CL>
int launch_image(const ImgArgs& A, int max_clusters, cudaStream_t stream) {
  using Gm = ImgGeom<N, CL>;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(image_kernel<N, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Gm::SMEM) != cudaSuccess)
      return DSB_E_CUDA;
    configured = true;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int n_clusters = sms / CL;
  if (max_clusters > 0) n_clusters = std::min(n_clusters, max_clusters);
  n_clusters = std::max(1, std::min(n_clusters, A.n_f * A.n_t));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(n_clusters * CL);
  cfg.blockDim = dim3(Gm::THREADS);
  cfg.dynamicSmemBytes = Gm::SMEM;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, image_kernel<N, CL>, A) != cudaSuccess) return DSB_E_CUDA;
  return launch_status();
}

}  // namespace

extern "C" {

int dsb_image_cluster_size(int n_grid) {
  switch (n_grid) {
    case 64: return 1;
    case 256: return 2;
    default: return 0;
  }
}

int dsb_image_fft(const void* D, long long d_rows, long long d_mask, const int* sc_off,
                  const void* sc_meta, const int* d_base, const int* n_filled,
                  const int* sfine, const int* f2c, const void* twiddles, int f0, int n_f, int G,
                  int N, long long t0, int n_t, int fftshift, void* out, int max_clusters,
                  int* status, cudaStream_t stream) {
  if (!D || !sc_off || !sc_meta || !d_base || !n_filled || !sfine || !f2c ||
      !twiddles || !out || n_f <= 0 || n_t <= 0 || G <= 0 || G > 48)
    return DSB_E_ARG;
  ImgArgs A{(const float2*)D, d_rows, d_mask, sc_off, (const int2*)sc_meta, d_base, n_filled, sfine,
            f2c, (const float2*)twiddles, f0, n_f, G, t0, n_t, fftshift, (float*)out, status};
  switch (N) {
    case 64: return launch_image<64, 1>(A, max_clusters, stream);
    case 256: return launch_image<256, 2>(A, max_clusters, stream);
    default: return DSB_E_UNSUPPORTED;
  }
}

}  // extern "C"
