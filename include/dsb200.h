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
#define DSB_E_BOUNDS 6       /* bounds-checked build: a table index out of  */
                             /* range (status; the access was skipped)      */

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
 * V[bls(a,b)] = sum conj(E_b) E_a, b <= a (F18).  On the tcgen05 tensor
 * cores, float32 accumulators in tensor memory, as the reference's fp16
 * HMMA correlator (src/dsart/services/triton_corr_fused.py:135-138): int8
 * codes and float16 voltages as kind::f16 (int8 -> f16 is exact, so integer
 * codes correlate exactly below 2^24), float32 voltages as kind::tf32 (each
 * part rounded to tf32, nearest, ties away).  nant <= 128.  status (device
 * int, may be null) receives DSB_E_TIMEOUT if a bounded wait gave up. */
int dsb_corr_split(const void* re, const void* im, int in_dtype, int nchan, int npkt, int nant,
                   int t_int, int fuse_stokes_i, int csf, void* out, int* status,
                   cudaStream_t stream);

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
 * channel.  Group (g, s) owns rows [yoff[g*ceff+s], + ycnt[...]); row r sums
 * the baselines row_bls[row_off[r] .. row_off[r+1]) (exact int32).
 * Output row r, tile f -> yout[((t_base + f) & t_mask)*y_t_stride + r]
 * (time-major ring; y_t_stride >= number of rows).
 * gains (may be null): (n_chgroup, ceff, nant) complex64, the gain of each
 * antenna in each summed channel; every visibility is multiplied by
 * g_a conj(g_b) before it is gridded (each product and sum rounded in
 * float32, rows summed in CSR order), the identity calibrated voltages
 * give (apply_cal_split, src/dsart/services/slow_corr_kernel.py:459)
 * when a gain is the same on the summed channels and both pols. */
int dsb_corr_tc_grid(const void* raw, long long raw_g_stride, int n_chgroup, int npkt, int nant,
                     int nchan, int t_int, int csf, const int* yoff, const int* ycnt,
                     const int* row_off, const int* row_bls, void* yout, long long y_t_stride,
                     long long t_base, long long t_mask, int max_ctas, const void* gains,
                     int* status, cudaStream_t stream);

/* ---- a6: uv cells in FP64 -------------------------------------------------
 * Replaces the (u, v) -> cell arithmetic of build_pattern / from_pattern
 * (src/dsart/grid/sparsity_pattern.py:1090-1170, grid/kernel.py:344-374):
 * col = rint(-(du/wl)/cell)+N/2, row = rint(-(dv/wl)/cell)+N/2,
 * wl = c/(nu*1e9); outputs (n_bl, n_ch) int32 row-major. */
int dsb_uv_cells(const double* du, const double* dv, int n_bl, const double* nu_ghz, int n_ch,
                 double cell_lambda, int n_grid, int* row, int* col, cudaStream_t stream);

/* ---- a7: gridder ----------------------------------------------------------
 * Replaces FastVisGridder.compute (src/dsart/grid/kernel.py:508-611), K=1:
 * out[f, cell] = sum over CSR sources (flat bls*C + s) of vis[f, src]. */
int dsb_grid_vis(const void* vis, int n_fv, long long nsrc, const int* cell_off,
                 const int* cell_src, int n_filled, void* out, cudaStream_t stream);

/* ---- a8: stage-1 shift + grid on visibilities ------------------------------
 * Replaces Stage1MultiDMCoarseDM._dedisperse_one_window
 * (src/dsart/services/corr_fast_integration.py:727-915) and the fused
 * Triton dedisp kernel (src/dsart/services/triton_dedisp.py:104):
 * out[d, t, cell] = sum_src vis_joined[t + shift[s, d], src], vis_joined =
 * prev[0:n_prev] ++ cur along time (the F34 sliding window). */
int dsb_dedisp_vis(const void* prev, const void* cur, int n_prev, long long nsrc, int ceff,
                   const int* cell_off, const int* cell_src, const int* shifts, int n_dm,
                   int n_filled, int t_dedisp, void* out, cudaStream_t stream);

/* ---- a9: static-sky mean ----------------------------------------------------
 * Replaces StaticSkyMean.apply (src/dsart/services/corr_fast_integration.py:1049-1240).
 * ring: (n_cells, window) float64 complex block means. */
int dsb_static_sky(const void* in, void* out, int n_t, int n_cells, void* ring, int window,
                   int head, int count, int subtract, cudaStream_t stream);

/* ---- a10: stage-2 aligned cube ----------------------------------------------
 * Replaces the slice assembly of Stage2InterChgroupShiftFifo.push
 * (src/dsart/coarse_dm/stage2_chgroup_alignment.py:264-338). hist[j] = device
 * pointer of the cube pushed j ticks ago. */
int dsb_stage2_roll(const void* const* hist, int depth, const int* kblk, const int* rsmp,
                    const int* warm, int n_dm, int t_len, long long inner, void* out,
                    cudaStream_t stream);

/* ---- a8-a10 pipeline form ---------------------------------------------------
 * Stage 1 over per-subband gridded rows (dsb_corr_tc_grid output), static-sky
 * subtraction fused, each output written at (t + shift2[g, d]) of the
 * stage-2 ring D, i.e. stage 1 + StaticSkyMean + the stage-2 FIFO
 * (corr_fast_integration.py:917, :1049; stage2_chgroup_alignment.py:264).
 * Rings are time-major with dense rows of pitch p[g] (a multiple of 4) per
 * chgroup:
 *   Y[(t & y_mask)*y_rows + y_base[g] + s*p[g] + cell]   (subband s),
 *   D[seg_base[gd] + (t mod seg_depth[gd])*p[g] + cell]  (gd = g*n_dm + d),
 * each (chgroup, coarse DM) its own ring segment of seg_depth[gd] (>= 8)
 * time slots, deep enough for its own stage-2 delay; the float64 sky ring
 * of (g, d, cell) is row d_base[g] + d*p[g] + cell.  y_base and y_rows are
 * multiples of 4, seg_base multiples of 4, Y and D 16-byte aligned (four
 * cells per access; pad cells up to the pitch).  d_bf16 selects the ring's
 * element: 0 = complex64; 1 = the BF16 storage form, one 32-bit word per
 * cell holding the real part (bf16, rounded to nearest even from the float32
 * sum) in the low half and the imaginary part in the high half; sums and the
 * sky statistics stay float32/float64.  amax, when not null, holds one
 * float per (chgroup g, coarse DM d) at g*n_dm + d, each raised (atomic
 * max) to the largest |part| of the float32 values written for it (the
 * bound dsb_image_fft sums under).  Block b covers cells
 * [blk_c0[b], + dsb_stage1_block_size()) of chgroup blk_g[b] and one group
 * of dm_group coarse DMs (grid y). */
int dsb_stage1_rows(const void* Y, long long y_rows, long long y_mask, int n_blocks,
                    const int* blk_g, const int* blk_c0, const int* y_base, const int* pitch,
                    const int* shift1, const int* shift2, const int* d_base, const int* n_filled,
                    void* D, int d_bf16, const long long* seg_base, const int* seg_depth,
                    float* amax, long long t0, int n_t, int n_dm, int ceff, int dm_group,
                    int max_spread,
                    void* sky_ring, int sky_window,
                    int sky_head, int sky_count, int sky_subtract, int* status,
                    cudaStream_t stream);
/* Cells per block (blk_c0 multiples of it); the largest DM group (coarse
 * DMs per block: 32, 16 or 8, grid y = ceil(n_dm / dm_group)); and the
 * shared memory a block needs for a DM group whose largest shift spread is
 * max_spread = the largest (max - min) of shift1[g, s, d] over the DMs of
 * one group (d in [k*group, (k+1)*group)).  The caller picks the largest
 * group that fits the device's 227 KB per block (a wide DM range over few
 * coarse DMs needs a smaller group); a spread larger than the one passed
 * sets DSB_E_CAPACITY in *status.  dsb_stage1_smem_bytes returns -1 for an
 * unsupported group or ceff. */
int dsb_stage1_block_size(void);
int dsb_stage1_dm_group(void);
long long dsb_stage1_smem_bytes(int ceff, int dm_group, int max_spread);
/* ---- a12: fine-DM combine ---------------------------------------------------
 * Pipeline form of combine_chgroups (src/dsart/fine_dm/combiner.py:548) with
 * the Hermitian half-spectrum fold and fftshift checkerboard of
 * fused_dequant_combine_per_fdm_half (src/dsart/image/fused_combine_cuda.py:560-620):
 * reads the segmented stage-2 ring directly (value of (g, coarse DM c,
 * cell) at time t: D[seg_base[g*n_coarse + c] + (t mod seg_depth[...])*d_pitch[g]
 * + cell]) and writes (n_f, n_t, N, N/2+1) complex64.  d_format names the
 * ring's element: 0 complex64 and 1 the BF16 storage form, as dsb_stage1_rows
 * writes them; 2 the cint8 wire form as dsb_ring_encode_cint8 writes it (int8
 * re in the low byte, im in the high byte of 16 bits; value float32(scale *
 * q) with the row's scale at scales[sc_base[g*n_coarse + c] + slot], slot the
 * time's ring slot).  scales and sc_base may be null for formats 0 and 1. */
int dsb_combine_rows(const void* D, int d_format, const long long* seg_base, const int* seg_depth,
                     const float* scales, const long long* sc_base, int n_coarse,
                     const int* hc_off, const int* e_g, const int* e_cell, const int* d_pitch,
                     const int* sfine, const int* f2c, int f0, int n_f, int G, int N,
                     long long t0, int n_t, int fftshift, void* out, cudaStream_t stream);

/* Reference-layout combine on dense cint8 streams [G, T, 2, N, N]: replaces
 * fused_dequant_combine_per_fdm[_half] and the calibrated variants
 * (src/dsart/image/fused_combine_cuda.py:1104, :1359; kernels :210-700).
 * scales/off_* null -> integer path; otherwise each term is scale * q +
 * offset (float32 fma, then add) with one value per chgroup [G], or, when
 * per_t != 0, per (chgroup, source time) [G, t_stream]: the per-tile scales
 * of the wire format (fused_combine_cuda.py:431-505).  out complex32
 * (out_f16) or complex64. */

/* ---- next row: RFI excision hook -------------------------------------------
 * Replaces apply_rfi_mask_to_voltages (src/dsart/services/
 * corr_fast_integration.py:1249-1370), applied to the raw on-wire pages
 * before the correlator instead of to the unpacked voltages: in raw
 * (n_pages, npkt, nant, nchan, 2t, 2p) uint8 (4-byte aligned), every sample
 * flagged in mask (n_pages, nant, nchan, 2) or, for packets of accumulation
 * a = pkt / (npkt / n_acc), in time_mask (n_pages, n_acc, nchan, 2) is set
 * to 0 (0 + 0i); nonzero flag bytes mean flagged; either mask may be null.
 * In place. */
int dsb_rfi_zero_fill(void* raw, int n_pages, int npkt, int nant, int nchan,
                      const unsigned char* mask, const unsigned char* time_mask, int n_acc,
                      cudaStream_t stream);

/* ---- next row: wire encoding of dedispersed rows ------------------------------
 * Replaces TransportTx._encode_rows (src/dsart/transport/tx.py:825-873).
 * rows: n_rows x n_filled complex64 cells, row r at rows + r*row_stride
 * (elements).  bits_per_cell 16: payload int8 (n_rows, n_filled, 2), per-row
 * scale = float32(amax / 127) over |re|, |im| (1 for an all-zero row),
 * q = clip(rint(x * float32(1 / scale)), -128, 127), ties to even.
 * bits_per_cell 32: payload half (n_rows, n_filled, 2), nearest-even,
 * scale 1.  Rows holding NaN or infinity are outside the reference's pinned
 * behaviour (its float-to-int8 conversion of them is platform-defined). */
int dsb_encode_rows(const void* rows, long long row_stride, int n_rows, int n_filled,
                    int bits_per_cell, void* payload, float* scales, cudaStream_t stream);
/* The same cint8 encoder applied to one chunk of stage-1 output, written
 * straight into the stage-2 ring, so that the ring holds what the search
 * side of the reference receives (TransportTx._encode_rows, tx.py:825-873,
 * per (chgroup, coarse DM, time) row, then the stage-2 FIFO).
 * X: complex64 (16-byte aligned); row (g, d, t), t in [0, n_t), at
 * X + x_base[g*n_dm + d] + t * pitch[g] with n_filled[g] pattern cells.
 * D: int8 pairs (4-byte aligned), row written at slot (t0 + t +
 * shift2[gd]) mod seg_depth[gd] of segment seg_base[gd] (cells past
 * n_filled set to 0); the row's scale at scales[sc_base[gd] + slot].
 * pitch, x_base and seg_base even (two cells per access); a row that breaks
 * this sets DSB_E_ARG in *status and is skipped. */
int dsb_ring_encode_cint8(const void* X, const long long* x_base, int n_t, const int* pitch,
                          const int* n_filled, int G, int n_dm, const int* shift2, long long t0,
                          void* D, const long long* seg_base, const int* seg_depth,
                          float* scales, const long long* sc_base, int* status,
                          cudaStream_t stream);
/* ---- a12: compact-layout combine -----------------------------------------------
 * combine_sparse_v4 (src/dsart/image/tiled_combine_cuda.py:1142; kernel :966)
 * with build_sparse_cell_csr's tables (:1092): dense [n_sb][n_filled_max]
 * [t_pad][re, im] int8 (time-minor compact streams, 2-byte aligned); the
 * n_act active half cells cell_uw = u * (N/2+1) + w with their entries
 * [cell_ptr[a], cell_ptr[a+1]) (at most 64 per cell) of stream ent_g
 * carrying the cell at compact index ent_k and / or its mirror at ent_km
 * (-1 where absent).  out[f][out_row0 + t][u][w] for t < t_out_len =
 * 0.5 (sum q(k) + conj q(km)) over the entries at stream time
 * t + t_lo - shifts[f * n_sb + g] (absent outside [0, t_rows)), times
 * (-1)^(u+w) if fftshift; int32 sums (exact), then half2 (out_f16) or
 * complex64.  Writes only the active cells: the caller zeroes the rest.
 * out is [n_fdm][out_rows][N][N/2+1].  A cell with more than 64 entries
 * sets DSB_E_CAPACITY in *status, an entry outside the tables DSB_E_ARG. */
int dsb_combine_sparse(const void* dense, const int* cell_uw, const int* cell_ptr,
                       const int* ent_g, const int* ent_k, const int* ent_km, int n_act,
                       const int* shifts, void* out, int out_f16, int n_sb, int t_rows,
                       int t_pad, int n_filled_max, int N, int n_fdm, int t_out_len, int t_lo,
                       int fftshift, int out_rows, int out_row0, int* status,
                       cudaStream_t stream);
int dsb_combine_dense(const void* streams, const int* shifts, const float* scales,
                      const float* off_re, const float* off_im, int per_t, void* out,
                      int out_f16, int half,
                      int G, int t_stream, int t_det, int N, int t_lo, int fftshift,
                      cudaStream_t stream);

/* ---- a12/a13: fused combine + 2-D inverse real FFT ------------------------------
 * Replaces fused_dequant_combine_per_fdm_half + torch.fft.irfft2 inside
 * GpuImager.process_cube (src/dsart/image/fused_combine_cuda.py:1359,
 * src/dsart/image/imager_gpu.py:575-605): for each (fine DM f0+fl, time t0+t)
 * the Hermitian half spectrum is combined from the segmented stage-2 ring
 * (as dsb_combine_rows reads it, in any of its three element forms; cint8
 * needs D 4-byte aligned) and
 * transformed on chip; out (n_f, n_t, N, N) float32 = irfft2(G_h) with
 * 1/N^2 normalisation (fftshifted when fftshift != 0).
 * Tables (built once per pattern set):
 *   S: the n_s distinct non-zero half cells (u, w), w in [0, N/2], sorted by
 *      (packed column w' = (w == N/2 ? 0 : w), n', u div LC, w == N/2) with
 *      n' = u mod LC, LC = N / fold; a slot is one (w', n');
 *   c_meta[cell_base[g] + k] = s | conj << 16 | g << 17: pattern cell k <
 *      n_filled[g] of chgroup g adds its value (conjugated if conj) to S
 *      entry s; each chgroup's run is padded with 0xffffffff to a multiple
 *      of 64 entries (cell_base[g] multiples of 64);
 *   c2[i] = {k | g << 16, s | conj << 16}: second targets (cells on w = 0 or
 *      w = N/2 that also land on their mirror);
 *   thr_b: (threads + 1) S ranges, one per kernel thread, each made of whole
 *      slots and at most max_entries long;
 *   gmeta, 16-byte aligned, in the form of meta_bits:
 *      16: (max_entries / 8, threads, 8) uint16, entry i of thread t at
 *      [i / 8][t][i % 8] = w' | n' << 7 | (u div LC) << 13 | (last entry of
 *      its slot) << 15;
 *      32: (max_entries / 4, threads, 4) uint32, entry i of thread t at
 *      [i / 4][t][i % 4] = w' | n' << 8 | (u div LC) << 14 | last << 17 |
 *      (w == N/2) << 18 | ((u + w) & 1) << 19; then, in the same buffer,
 *      the fold's compact tables: (max_entries / 8, threads) uint32 with
 *      entry i's nibble (u div LC) | last << 3 at bits 4 (i % 8) of word
 *      [i / 8][t]; (threads + 1) int32 first slot of each thread (the slots
 *      in S order), padded to 16 bytes; (threads, 4) uint32 with entry i's
 *      (w == N/2) | ((u + w) & 1) << 1 at bits 2 (i % 16) of word [t][i / 16];
 *      one uint16 per slot, n' * (N/2 + 2) + w', padded to 8 entries;
 *   srot (16-bit form only; may be null for the 32-bit form): (threads)
 *      uint64, 2 bits per entry i at bit 2i: (w == N/2) | ((u + w) & 1) << 1;
 *   dcols/dmask: the n_dense packed columns with an entry off n' = 0 and
 *      the bit mask of their occupied n';
 *   kcols: the n_const other packed columns, w' | (has entries) << 16;
 *      n_dense + n_const = N/2, every packed column once.
 *   s_mult: the most contributions (c_meta and c2 entries) to one S entry.
 * Sums: S is summed in int32 fixed point, each part times 2^k rounded to an
 * integer, so the sum does not depend on the order of the adds.  k comes
 * from a bound on the image's parts: for the cint8 form the rows' scales
 * (k = 22 - ilogb(max scale) - ceil(log2(s_mult))); for forms 0 and 1 the
 * bound rows stage 1 keeps (dsb_stage1_rows' amax), row (floor(t1 /
 * amax_chunk) mod amax_rows) of (amax_rows, G * n_coarse) floats for the
 * value of stage-1 time t1 = t - sfine - shift2[g*n_coarse + c]
 * (k = 28 - ilogb(max bound) - ceil(log2(s_mult))).  A part's rounding
 * error is at most 2^-(k+1), below 2^(ceil(log2(s_mult)) - 29) of the bound;
 * bf16 parts above 2^-16 of it are exact.  k is clamped at 100 (so that
 * 2^-k x 0.5/N^2 stays a normal float): bounds below about 2^-72 get a
 * coarser grid.  The bound must cover every value
 * read: the caller keeps a row alive while the ring holds its chunk and
 * zeroes it before stage 1 writes a new chunk into it.  A non-finite bound
 * sets DSB_E_ARG in *status.
 * twiddles: (N) complex64 exp(+2 pi i e/N).  Supported N: 64, 256, 512; n_s
 * must fit the kernel's S capacity (s_capacity of dsb_image_geometry) or
 * DSB_E_CAPACITY is returned.  status: a thread range longer than
 * max_entries or a cell_base[g] that is not a multiple of 64 sets
 * DSB_E_CAPACITY and writes nothing.  Each CTA holds 128 columns of tensor
 * memory while it runs (all 512 of its SM at N = 512). */
/* Dense inverse real 2-D FFT, the torch.fft.irfft2(half, s=(N, N)) that
 * GpuImager.process_cube runs after its dense combine
 * (src/dsart/image/imager_gpu.py:590): half [n_img][N][N/2+1] complex64 ->
 * out [n_img][N][N] float32, 1/N^2 normalisation, the imaginary parts of
 * columns 0 and N/2 dropped after the column transforms (as numpy and cuFFT
 * do).  half is used as the work buffer and is overwritten.  twiddles: (N)
 * complex64 exp(+2 pi i e/N).  N in {32, 64, 128, 256, 512}; n_img <= 65535. */
int dsb_irfft2(void* half, int n_img, int N, const void* twiddles, float* out,
               cudaStream_t stream);

/* The kernel's geometry at grid size n_grid, for building the tables above:
 * geom[0] fold (column passes, LC = N / fold), geom[1] threads per CTA,
 * geom[2] max_entries (S entries per thread), geom[3] meta_bits (16 or 32),
 * geom[4] s_capacity.  DSB_E_UNSUPPORTED for any other n_grid.  No
 * counterpart in the reference (a query for the tables of dsb_image_fft). */
int dsb_image_geometry(int n_grid, int* geom);
int dsb_image_fft(const void* D, int d_format, const long long* seg_base, const int* seg_depth,
                  const float* scales, const long long* sc_base, const float* amax,
                  const int* shift2, int amax_chunk, int amax_rows, int n_coarse,
                  const unsigned* c_meta, const int* cell_base, const void* c2, int n_c2,
                  const int* thr_b, const void* gmeta, const unsigned long long* srot, int n_s,
                  int s_mult, const int* dcols, const unsigned long long* dmask, int n_dense,
                  const int* kcols, int n_const, const int* d_pitch, const int* n_filled,
                  const int* sfine, const int* f2c, const void* twiddles, int f0, int n_f, int G,
                  int N, long long t0, int n_t, int fftshift, void* out, int max_blocks,
                  int* status, cudaStream_t stream);

/* ---- a13/a14: edge mask x Layer-1 normalisation into the detector cube -----
 * Replaces the mask multiply + cube write of GpuImager.process_cube
 * (src/dsart/image/imager_gpu.py:604-650): cube[t, f0+f, p] = img[f, t, p] *
 * mask[(f,) p]. */
int dsb_mask_to_cube(const float* img, const float* mask, int mask_per_f, int n_f, int n_t,
                     int npix, void* cube, int cube_f16, int cube_f_total, int cube_f0,
                     cudaStream_t stream);

/* ---- a15: boxcar detector ----------------------------------------------------
 * precompute_padded_cumsum (src/dsart/detector/forward.py:250): float64
 * running prefix rounded to float32, max_w//2 zero rows on the left,
 * max_w-1-max_w//2 copies of the last prefix on the right. */
int dsb_padded_cumsum(const void* x, int x_f16, int n, long long inner, int max_w, float* cs,
                      cudaStream_t stream);

/* multi_boxcar_argmax_triton (src/dsart/detector/triton_boxcar.py:305, kernel
 * :193): snr_k = (cs[t+off_k+w_k] - cs[t+off_k]) * sigma_inv_k, strict '>'. */
int dsb_multi_boxcar_argmax(const float* cs, long long inner, const int* widths,
                            const int* offsets, const float* sigma_inv, int K, int n_out,
                            int t_base, void* out_max, int out_f16, void* out_win,
                            cudaStream_t stream);

/* The two calls above in one, for callers that cannot allocate device memory
 * (a host that gives all of the GPU's memory to its own fixed arena, or a
 * real-time loop where an allocation or free would stall every stream on the
 * device).  No counterpart in dsa110-rt: it has no such callers.  The prefix
 * sums live in a fixed array inside the library, DSB_NOALLOC_SCRATCH_BYTES
 * long, held on every GPU that loads the library until the process exits;
 * (n + max_w) * inner * 4 bytes beyond it return DSB_E_CAPACITY (computed in
 * 64 bits, so no n, max_w or inner can wrap past the check).  The first
 * call in each CUDA context looks up that array's address (cached per
 * context ID, so a cudaDeviceReset or another context gets its own lookup),
 * so make it before any stream capture.  Every call shares the one array:
 * calls that overlap on the GPU (two streams, or two host threads) race and
 * must be serialised by the caller.  Needs t_base + n_out <= n and the
 * centred offsets max_w/2 - widths[k]/2 with widths[k] <= max_w; an output
 * whose widths / offsets would read a prefix row outside this call's
 * n + max_w rows gets S/N NaN and winner -1 (nothing outside is read).
 * Allocates nothing. */
#define DSB_NOALLOC_SCRATCH_BYTES (16u << 20)
int dsb_boxcar_argmax_noalloc(const void* x, int x_f16, int n, long long inner, int max_w,
                              const int* widths, const int* offsets, const float* sigma_inv,
                              int K, int n_out, int t_base, void* out_max, int out_f16,
                              void* out_win, cudaStream_t stream);

/* boxcar_from_padded_cumsum (src/dsart/detector/forward.py:339). */
int dsb_boxcar_from_cs(const float* cs, long long inner, int width, int start, int n_out,
                       float* out, cudaStream_t stream);

/* Fused streaming form of the three above plus the threshold test of
 * decode_topk_argmax_lowmem (src/dsart/detector/decoder.py:388): widths
 * 1..2^log_maxw over n samples of n_f*npix cells; cell e = f*npix + p at time
 * t is read at cube[f*f_stride + t*t_stride + p] and multiplied by
 * mask[f*mask_f_stride + p] (the edge mask; mask_f_stride 0 shares one mask
 * over the fine DMs), divided by sig_f[f] (the Layer-1 sigma) when sig_f is
 * non-null.  Every output cell with max S/N > threshold is appended to
 * cands (struct {int t, pix; float snr; int k;}, pix = e + pix_off); count[0]
 * counts them (entries past cap are counted, not written; the count stops
 * growing a little above 2^30, so it never wraps, and cap may not exceed
 * 2^30) and count[1]
 * keeps the bits of the largest S/N that was not written (0 when every entry
 * fit): a caller selecting the top entries knows its selection is exact
 * when that S/N lies below them.  count points at two ints, zeroed before
 * the launch.  Float cubes whose npix is a multiple of 32 (16-byte aligned,
 * strides in whole 16-byte units) are staged into shared memory by TMA with
 * bounded waits: a wait that runs out leaves count[1] = 0x7fc00000 (a quiet
 * NaN, above any S/N's bits), which the caller reads as DSB_E_TIMEOUT. */
int dsb_detect(const void* cube, int cube_f16, int n, int n_f, int npix, long long f_stride,
               long long t_stride, const float* mask, long long mask_f_stride,
               const float* sig_f, int log_maxw, const float* sigma_inv, int t_base, int n_out,
               float threshold, void* cands, int cap, int pix_off, int* count,
               cudaStream_t stream);

/* dsb_detect plus the Layer-2 score subsample of the streaming detector
 * (DeterministicDetector._streaming_forward, src/dsart/detector/
 * forward.py:1425-1530; noise_norm/layer2.py:58): while it marches, the
 * detector writes the raw boxcar sum of width 2^k (before sigma_inv) of
 * every sampled (cell, output time) to l2_out[k * l2_m + slot].  l2_ent:
 * 16-byte aligned int4 entries {eg, t, k, slot} sorted by (eg, t), eg =
 * cell index + pix_off over all fine DMs, t = output time - t_base;
 * l2_off[gb]: first entry with eg >= 256 gb (one more entry at the end);
 * pix_off a multiple of 256.  Slots without an entry are not written (the
 * caller keeps the masked-out ones NaN, which the clipped std drops).  With
 * l2_out null this is dsb_detect. */
int dsb_detect_sampled(const void* cube, int cube_f16, int n, int n_f, int npix,
                       long long f_stride, long long t_stride, const float* mask,
                       long long mask_f_stride, const float* sig_f, int log_maxw,
                       const float* sigma_inv, int t_base, int n_out, float threshold,
                       void* cands, int cap, int pix_off, int* count, const int* l2_off,
                       const void* l2_ent, float* l2_out, int l2_m, cudaStream_t stream);

/* ---- a18: Layer-1 sigma-clipped std ---------------------------------------------
 * sigma_clipped_std_batched (src/dsart/noise_norm/layer1.py:53): rows of at
 * most 4096 samples; lower median; non-finite samples dropped. */
int dsb_clipped_std(const float* samples, int rows, int m, float n_sigma, int n_iter, float* out,
                    cudaStream_t stream);

/* Layer-1 sigma of each fine DM straight from the images, as
 * CubePipeline._layer1_normalise (src/dsart/services/cube_pipeline.py:2226)
 * with sigma_clipped_std_batched: row f's samples are img[f*f_stride +
 * times[i]*t_stride + pix[j]] for every (i, j) (n_times*n_pix <= 4096);
 * sigma[f] = the clipped std, or 1 where that is not > 0 (the mask divisor). */
int dsb_layer1_sigma(const float* img, long long f_stride, long long t_stride, int n_f,
                     const int* times, int n_times, const int* pix, int n_pix, float n_sigma,
                     int n_iter, float* sigma, cudaStream_t stream);

/* ---- the batched form: one block's launch sequence as a CUDA graph -------------
 * No counterpart in the reference (its per-group plain runs are Python
 * loops of launches).  dsb_graph_begin(stream) starts capturing (relaxed
 * mode) on a non-default stream; the launches made on it are recorded, not
 * run.  dsb_graph_end_launch(stream, &exec) ends the capture, instantiates
 * the graph into *exec the first time (exec null) or updates *exec in place
 * with the new graph's arguments (cudaGraphExecUpdate; a changed topology
 * is instantiated afresh), and launches it on the stream.
 * dsb_graph_abort(stream) ends a capture whose host side failed part-way
 * and discards it (nothing runs).  dsb_graph_destroy(exec) frees *exec. */
int dsb_graph_begin(cudaStream_t stream);
int dsb_graph_end_launch(cudaStream_t stream, void** exec);
int dsb_graph_abort(cudaStream_t stream);
int dsb_graph_destroy(void* exec);

/* ---- a3: per-antenna complex gains on split voltages ---------------------------
 * Replaces apply_cal_split (src/dsart/services/slow_corr_kernel.py:459-528,
 * eager form :417-423): out_re = re*g_re - im*g_im, out_im = re*g_im + im*g_re
 * on voltages (nchan, ntimes, npol, npkt, nant) with gains (gain_nchan, 1,
 * npol, 1, nant), gain_nchan 1 or nchan (broadcast), all contiguous, float16
 * (dtype_f16 = 1) or float32.  Rounded as the reference's eager tensor ops:
 * half products rounded to half, their sum / difference taken in float32
 * and rounded to half; float32 without fused multiply-adds.  Writes new
 * out_re, out_im (not in place). */
int dsb_cal_apply(const void* re, const void* im, const void* gain_re, const void* gain_im,
                  int dtype_f16, int nchan, int ntimes, int npol, int npkt, int nant,
                  int gain_nchan, void* out_re, void* out_im, cudaStream_t stream);

/* ---- next row: per-cube clusterer (host) ------------------------------------
 * The minimum spanning tree of the HDBSCAN backend that cluster/forward.py:103
 * runs through the hdbscan package: X (n, d) float64 row-major feature rows,
 * cityblock distances (summed over the columns in order), core[a] = the
 * min_samples-th smallest distance from a counting a itself as the 0-th
 * (min_samples clamped to [1, n - 1]), mutual reachability max(D, core_a,
 * core_b), Prim's algorithm from point 0 (first index on a tie, strict
 * improvement to update).  edges: (n - 1) x 3 doubles (source, point,
 * distance) in the order added.  Host code, no stream; n >= 2. */
int dsb_cluster_mst(const double* X, int n, int d, int min_samples, double* core,
                    double* edges);

#ifdef __cplusplus
}
#endif

#endif /* DSB200_H */
