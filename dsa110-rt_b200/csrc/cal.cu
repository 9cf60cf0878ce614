// Per-(channel, pol, antenna) complex gain on split real/imag voltages
// (sm_100a): apply_cal_split of the reference (services/slow_corr_kernel.py:
// 417-423, 459-528):
//   out_re = re * g_re - im * g_im
//   out_im = re * g_im + im * g_re
// on the GEMM layout (nchan, ntimes, npol, npkt, nant), with the gains in the
// broadcast layout (cal_nchan, 1, npol, 1, nant), cal_nchan 1 or nchan.
//
// Rounding follows the reference's eager torch ops, one tensor op at a time:
//   float16: each product rounded to half (the float32 product of two halves
//            is exact), then the sum or difference of the two halves taken in
//            float32 and rounded to half (torch's half arithmetic computes in
//            float32 and stores half);
//   float32: each product and the sum rounded to float32, no fused
//            multiply-add.
// Two antennas per thread (one 4- or 8-byte access) when nant is even.
#include "dsb_common.cuh"

#include <algorithm>

namespace {

int launch_status() { return cudaGetLastError() == cudaSuccess ? DSB_OK : DSB_E_CUDA; }

DSB_DEV __half cal_re_h(__half r, __half i, __half gr, __half gi) {
  const float a = __half2float(__hmul(r, gr)), b = __half2float(__hmul(i, gi));
  return __float2half_rn(a - b);
}
DSB_DEV __half cal_im_h(__half r, __half i, __half gr, __half gi) {
  const float a = __half2float(__hmul(r, gi)), b = __half2float(__hmul(i, gr));
  return __float2half_rn(a + b);
}
DSB_DEV float cal_re_f(float r, float i, float gr, float gi) {
  return __fsub_rn(__fmul_rn(r, gr), __fmul_rn(i, gi));
}
DSB_DEV float cal_im_f(float r, float i, float gr, float gi) {
  return __fadd_rn(__fmul_rn(r, gi), __fmul_rn(i, gr));
}

// element (ch, t, p, k, a) -> gain index (ch or 0, p, a)
DSB_DEV long long gain_index(long long e, int nant, int npkt, int npol, int ntimes, bool per_ch) {
  const long long a = e % nant;
  long long r = e / nant;
  r /= npkt;
  const long long p = r % npol;
  r /= npol;
  const long long ch = r / ntimes;
  return ((per_ch ? ch : 0) * npol + p) * nant + a;
}

template <typename T>
__global__ void __launch_bounds__(256) cal_apply_kernel(
    const T* __restrict__ re, const T* __restrict__ im, const T* __restrict__ gre,
    const T* __restrict__ gim, long long n, int nant, int npkt, int npol, int ntimes,
    int per_ch, T* __restrict__ ore, T* __restrict__ oim) {
  // two antennas (a, a + 1) per thread; nant is even
  const long long n2 = n / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2;
       j += (long long)gridDim.x * blockDim.x) {
    const long long e = 2 * j;
    const long long gi = gain_index(e, nant, npkt, npol, ntimes, per_ch != 0);
    if constexpr (sizeof(T) == 2) {
      const __half2 r = reinterpret_cast<const __half2*>(re)[j];
      const __half2 i = reinterpret_cast<const __half2*>(im)[j];
      const __half2 gr = *reinterpret_cast<const __half2*>(gre + gi);
      const __half2 gm = *reinterpret_cast<const __half2*>(gim + gi);
      reinterpret_cast<__half2*>(ore)[j] =
          __halves2half2(cal_re_h(__low2half(r), __low2half(i), __low2half(gr), __low2half(gm)),
                         cal_re_h(__high2half(r), __high2half(i), __high2half(gr), __high2half(gm)));
      reinterpret_cast<__half2*>(oim)[j] =
          __halves2half2(cal_im_h(__low2half(r), __low2half(i), __low2half(gr), __low2half(gm)),
                         cal_im_h(__high2half(r), __high2half(i), __high2half(gr), __high2half(gm)));
    } else {
      const float2 r = reinterpret_cast<const float2*>(re)[j];
      const float2 i = reinterpret_cast<const float2*>(im)[j];
      const float2 gr = *reinterpret_cast<const float2*>(gre + gi);
      const float2 gm = *reinterpret_cast<const float2*>(gim + gi);
      reinterpret_cast<float2*>(ore)[j] =
          make_float2(cal_re_f(r.x, i.x, gr.x, gm.x), cal_re_f(r.y, i.y, gr.y, gm.y));
      reinterpret_cast<float2*>(oim)[j] =
          make_float2(cal_im_f(r.x, i.x, gr.x, gm.x), cal_im_f(r.y, i.y, gr.y, gm.y));
    }
  }
}

// one antenna per thread (odd nant)
template <typename T>
__global__ void __launch_bounds__(256) cal_apply_scalar_kernel(
    const T* __restrict__ re, const T* __restrict__ im, const T* __restrict__ gre,
    const T* __restrict__ gim, long long n, int nant, int npkt, int npol, int ntimes,
    int per_ch, T* __restrict__ ore, T* __restrict__ oim) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long gi = gain_index(e, nant, npkt, npol, ntimes, per_ch != 0);
    if constexpr (sizeof(T) == 2) {
      ore[e] = cal_re_h(re[e], im[e], gre[gi], gim[gi]);
      oim[e] = cal_im_h(re[e], im[e], gre[gi], gim[gi]);
    } else {
      ore[e] = cal_re_f(re[e], im[e], gre[gi], gim[gi]);
      oim[e] = cal_im_f(re[e], im[e], gre[gi], gim[gi]);
    }
  }
}

}  // namespace

extern "C" {

int dsb_cal_apply(const void* re, const void* im, const void* gain_re, const void* gain_im,
                  int dtype_f16, int nchan, int ntimes, int npol, int npkt, int nant,
                  int gain_nchan, void* out_re, void* out_im, cudaStream_t stream) {
  if (!re || !im || !gain_re || !gain_im || !out_re || !out_im || nchan <= 0 || ntimes <= 0 ||
      npol <= 0 || npkt <= 0 || nant <= 0 || (gain_nchan != 1 && gain_nchan != nchan))
    return DSB_E_ARG;
  const long long n = (long long)nchan * ntimes * npol * npkt * nant;
  const int per_ch = gain_nchan == nchan && nchan > 1;
  const size_t esz = dtype_f16 ? 2 : 4;
  const uintptr_t all = reinterpret_cast<uintptr_t>(re) | reinterpret_cast<uintptr_t>(im) |
                        reinterpret_cast<uintptr_t>(gain_re) |
                        reinterpret_cast<uintptr_t>(gain_im) |
                        reinterpret_cast<uintptr_t>(out_re) | reinterpret_cast<uintptr_t>(out_im);
  const bool pair = (nant % 2) == 0 && (all % (2 * esz)) == 0;
  const long long work = pair ? n / 2 : n;
  const int blocks = (int)std::max<long long>(1, std::min<long long>((work + 255) / 256, 148 * 32));
#define DSB_CAL(K, T)                                                                       \
  K<T><<<blocks, 256, 0, stream>>>((const T*)re, (const T*)im, (const T*)gain_re,           \
                                   (const T*)gain_im, n, nant, npkt, npol, ntimes, per_ch,  \
                                   (T*)out_re, (T*)out_im)
  if (dtype_f16) {
    if (pair) DSB_CAL(cal_apply_kernel, __half);
    else DSB_CAL(cal_apply_scalar_kernel, __half);
  } else {
    if (pair) DSB_CAL(cal_apply_kernel, float);
    else DSB_CAL(cal_apply_scalar_kernel, float);
  }
#undef DSB_CAL
  return launch_status();
}

}  // extern "C"
