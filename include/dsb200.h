/*
 * dsb200 — C ABI of the B200 (sm_100a) implementation of dsa110-rt's fast
 * FRB-search hot path.
 *
 * Every entry point takes plain device pointers, sizes and strides plus the
 * CUDA stream to launch on, returns DSB_OK (0) or a DSB_E_* code before any
 * launch on a bad argument, and never allocates device memory: callers own
 * every buffer (the Python layer uses torch tensors).  Kernels that can give
 * up (a bounded wait that ran out) record a code in the optional device
 * `status` word; callers read it after the stream synchronises.
 *
 * Each declaration names the dsa110-rt interface it replaces (path:line in
 * the dsa110-rt project).
 */
#ifndef DSB200_H
#define DSB200_H

#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSB_VERSION 1

#define DSB_OK 0
#define DSB_E_ARG 1          /* invalid argument (shape, size, alignment)   */
#define DSB_E_CUDA 2         /* CUDA launch or runtime error                */
#define DSB_E_UNSUPPORTED 3  /* geometry outside what the kernel supports   */
#define DSB_E_TIMEOUT 4      /* device-side bounded wait ran out (status)   */
#define DSB_E_CAPACITY 5     /* a size exceeds a fixed capacity             */

#define DSB_DT_INT8 0
#define DSB_DT_F16 1
#define DSB_DT_F32 2

int dsb_version(void);
const char* dsb_strerror(int code);

/* ---- a1: 4-bit unpack ---------------------------------------------------
 * Replaces unpack_int4_split (src/dsart/services/slow_corr_kernel.py:220) and
 * its Triton kernel (src/dsart/services/triton_unpack_onwire.py:51).
 * raw: on-wire (npkt, nant, nchan, 2t, 2p) bytes, low nibble = real, high =
 * imag, two's complement.  out_re/out_im: GEMM layout (nchan, 2t, 2p, npkt,
 * nant) of out_dtype (DSB_DT_*), value = code * scale (int8 ignores scale). */
int dsb_unpack_int4(const void* raw, int npkt, int nant, int nchan, int out_dtype, float scale,
                    void* out_re, void* out_im, cudaStream_t stream);

/* ---- a4: correlator on GEMM-layout voltages ------------------------------
 * Replaces FastCorrKernel.compute_split
 * (src/dsart/services/corr_fast_kernel.py:364-413, CPU path :698-755).
 * re/im: (nchan, 2t, 2p, npkt, nant) of in_dtype.  out (complex64):
 * fuse_stokes_i -> (n_fv, nbase, nchan/csf); else (n_fv, nbase, nchan, 2).
 * V[bls(a,b)] = sum conj(E_b) E_a, b <= a (F18). */
int dsb_corr_split(const void* re, const void* im, int in_dtype, int nchan, int npkt, int nant,
                   int t_int, int fuse_stokes_i, int csf, void* out, cudaStream_t stream);

/* ---- a4/a5: fused unpack + correlate on tcgen05 tensor cores -------------
 * Replaces the unpack -> cal -> fused HMMA correlator chain
 * (src/dsart/services/triton_unpack_onwire.py:164 +
 *  src/dsart/services/triton_corr_fused.py:155 via corr_fast_kernel.py:530)
 * for the Stokes-I + channel-sum product, integer exact.
 * raw: n_chgroup on-wire pages of (npkt, nant, nchan, 2, 2) bytes,
 * raw_g_stride bytes apart (16-byte aligned).  Output element
 * (g, f, bls, s) -> out[g*o_g + f*o_f + bls*o_b + s*o_s] (complex64).
 * unit_order: 0 walks fast-vis tiles fastest, 1 summed channels fastest
 * (choose the one whose output stride is smallest). */
int dsb_corr_tc(const void* raw, long long raw_g_stride, int n_chgroup, int npkt, int nant,
                int nchan, int t_int, int csf, int unit_order, void* out, long long o_g,
                long long o_f, long long o_b, long long o_s, int max_ctas, int* status,
                cudaStream_t stream);

/* Same correlator with the gridder folded into its epilogue: replaces
 * FastVisGridder.compute (src/dsart/grid/kernel.py:508) applied per summed
 * channel.  ycell[(g*ceff + s)*nbase + bls] = row within group (g, s) or -1;
 * group rows start at yoff[g*ceff+s] and number ycnt[...] (<= ymax).
 * Output row r, tile f -> yout[r*y_t_stride + ((t_base + f) & t_mask)]. */
int dsb_corr_tc_grid(const void* raw, long long raw_g_stride, int n_chgroup, int npkt, int nant,
                     int nchan, int t_int, int csf, const int* ycell, const int* yoff,
                     const int* ycnt, int ymax, void* yout, long long y_t_stride,
                     long long t_base, long long t_mask, int max_ctas, int* status,
                     cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* DSB200_H */
