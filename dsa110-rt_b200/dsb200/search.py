"""Search side: fine-DM combine, imaging, boxcar detector, Layer-1 noise —
drop-in for ``dsart.image.fused_combine_cuda`` (fused_dequant_combine_per_fdm
:1104, ``_half`` :1359), ``dsart.image.imager`` (compute_edge_mask :112,
image_mask_npad :57), ``dsart.detector.forward`` (precompute_padded_cumsum
:250, boxcar_from_padded_cumsum :339), ``dsart.detector.triton_boxcar``
(multi_boxcar_argmax_triton :305), ``dsart.detector.decoder``
(decode_topk_argmax_lowmem :388) and ``dsart.noise_norm.layer1``
(sigma_clipped_std_batched :53).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np
import torch

from . import _lib

# ---------------------------------------------------------------------------
# combine (reference dense cint8 layout)
# ---------------------------------------------------------------------------


def _combine_dense(streams_cint8, shifts, output, *, half, scales, offsets_re, offsets_im,
                   t_lo, fftshift):
    for t, nm in ((streams_cint8, "streams_cint8"), (shifts, "shifts"), (output, "output")):
        _lib.require_cuda(t, nm)
    if streams_cint8.dtype != torch.int8 or streams_cint8.ndim != 5 or streams_cint8.shape[2] != 2:
        raise RuntimeError(f"streams_cint8 must be int8 [G, T, 2, N, N]; got "
                           f"{streams_cint8.dtype} {tuple(streams_cint8.shape)}")
    G, T, _, N, N2 = streams_cint8.shape
    if N != N2:
        raise RuntimeError("streams_cint8 grid must be square")
    if shifts.dtype != torch.int32 or shifts.shape != (G,):
        raise RuntimeError(f"shifts must be int32 ({G},)")
    nw = N // 2 + 1 if half else N
    if output.ndim != 3 or output.shape[1:] != (N, nw):
        raise RuntimeError(f"output must be [T_det - t_lo, {N}, {nw}]; got {tuple(output.shape)}")
    if output.dtype not in (torch.complex32, torch.complex64):
        raise RuntimeError(f"output dtype {output.dtype} not in (complex32, complex64)")
    calib = scales is not None
    # per-(chgroup, source time) scales [G, T] (the wire's per-tile scales) when
    # all three are 2-D, as fused_combine_cuda.py:1299-1330 decides
    per_t = calib and all(t is not None and t.dim() == 2
                          for t in (scales, offsets_re, offsets_im))
    if calib:
        want = (G, T) if per_t else (G,)
        for t, nm in ((scales, "scales"), (offsets_re, "offsets_re"), (offsets_im, "offsets_im")):
            if t is None or t.dtype != torch.float32 or tuple(t.shape) != want:
                raise RuntimeError(f"{nm} must be float32 {want}")
            _lib.require_cuda(t, nm)
            if not t.is_contiguous():
                raise RuntimeError(f"{nm} must be contiguous")
    t_det = int(t_lo) + int(output.shape[0])
    _lib.check(_lib.lib().dsb_combine_dense(
        _lib.ptr(streams_cint8), _lib.ptr(shifts), _lib.ptr(scales if calib else None),
        _lib.ptr(offsets_re if calib else None), _lib.ptr(offsets_im if calib else None),
        int(per_t), _lib.ptr(output), int(output.dtype == torch.complex32), int(half), G, T, t_det, N,
        int(t_lo), int(bool(fftshift)), _lib.stream_of(output.device)), "dsb_combine_dense")


def fused_dequant_combine_per_fdm(streams_cint8, shifts, output, *, scales=None, offsets_re=None,
                                  offsets_im=None, t_lo: int = 0, fftshift: bool = True) -> None:
    """Full-grid combine into ``output [T_det - t_lo, N, N]`` (fused_combine_cuda.py:1104)."""
    _combine_dense(streams_cint8, shifts, output, half=False, scales=scales,
                   offsets_re=offsets_re, offsets_im=offsets_im, t_lo=t_lo, fftshift=fftshift)


def fused_dequant_combine_per_fdm_half(streams_cint8, shifts, output, *, scales=None,
                                       offsets_re=None, offsets_im=None, t_lo: int = 0,
                                       fftshift: bool = True) -> None:
    """Hermitian half-spectrum combine into ``[T_det - t_lo, N, N/2+1]``
    (fused_combine_cuda.py:1359)."""
    _combine_dense(streams_cint8, shifts, output, half=True, scales=scales,
                   offsets_re=offsets_re, offsets_im=offsets_im, t_lo=t_lo, fftshift=fftshift)


# ---------------------------------------------------------------------------
# combine (compact time-minor layout; tiled_combine_cuda.py:1080-1240)
# ---------------------------------------------------------------------------

# per-cell stream-count buckets, the reference's launch grouping (:1069)
_V4_BUCKETS = (8, 16, 32, 64)


@dataclass
class SparseCellCsr:
    """Per-half-cell list of the streams carrying the cell or its mirror
    (tiled_combine_cuda.py:1069-1090): active cells ``cell_uw = u * (N/2+1)
    + w`` grouped by entry-count bucket (<= 8, 16, 32, 64) and ascending
    inside a bucket, entries [cell_ptr[a], cell_ptr[a+1]) with stream
    ``ent_g`` (ascending) and compact indices ``ent_k`` / ``ent_km`` of the
    cell and its mirror (-1 where absent); ``buckets`` (start, end, max
    entries) per non-empty bucket."""
    n_sb: int
    n_grid: int
    cell_uw: torch.Tensor
    cell_ptr: torch.Tensor
    ent_g: torch.Tensor
    ent_k: torch.Tensor
    ent_km: torch.Tensor
    buckets: tuple

    @property
    def n_cells(self) -> int:
        return int(self.cell_uw.shape[0])

    @property
    def n_entries(self) -> int:
        return int(self.ent_g.shape[0])


def build_sparse_cell_csr(inv_lut: torch.Tensor, *, n_grid: int) -> SparseCellCsr:
    """The tables of ``combine_sparse_v4`` from the inverse LUT ``[n_sb,
    N*N]`` (compact index of each grid cell in each stream, -1 if absent):
    tiled_combine_cuda.py:1092.  Built once per pattern set (host)."""
    n_sb = int(inv_lut.shape[0])
    N = int(n_grid)
    if tuple(inv_lut.shape) != (n_sb, N * N):
        raise ValueError(f"inv_lut must be (n_sb, {N * N}); got {tuple(inv_lut.shape)}")
    if n_sb > 64:
        raise ValueError(f"v4 supports n_sb <= 64; got {n_sb}")
    dev = inv_lut.device
    lut = inv_lut.detach().to("cpu").numpy().astype(np.int64)
    nh = N // 2 + 1
    u = np.repeat(np.arange(N), nh)
    w = np.tile(np.arange(nh), N)
    lin = u * N + w
    linm = ((N - u) % N) * N + ((N - w) % N)
    k_lin = lut[:, lin].T                   # [n_half_cells, n_sb]
    k_linm = lut[:, linm].T
    present = (k_lin >= 0) | (k_linm >= 0)
    ne = present.sum(1)
    uw = u * nh + w
    order_parts, buckets, lo, start = [], [], 0, 0
    for hi in _V4_BUCKETS:
        sel = np.flatnonzero((ne > lo) & (ne <= hi))
        if sel.size:
            order_parts.append(sel)
            buckets.append((start, start + int(sel.size), int(ne[sel].max())))
            start += int(sel.size)
        lo = hi
    order = np.concatenate(order_parts) if order_parts else np.zeros(0, np.int64)
    cell_ptr = np.zeros(order.size + 1, np.int32)
    cell_ptr[1:] = np.cumsum(ne[order])
    rows, g = np.nonzero(present[order])    # cell-major, g ascending
    cells = order[rows]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(dev)  # noqa: E731
    return SparseCellCsr(n_sb=n_sb, n_grid=N, cell_uw=t(uw[order]), cell_ptr=t(cell_ptr),
                         ent_g=t(g), ent_k=t(k_lin[cells, g]), ent_km=t(k_linm[cells, g]),
                         buckets=tuple(buckets))


def combine_sparse_v4(dense: torch.Tensor, csr: SparseCellCsr, shifts: torch.Tensor, *,
                      t_rows: int, t_out_len: int, t_lo: int = 0, fftshift: bool = True,
                      threads: int = 512, out: torch.Tensor, out_row0: int = 0,
                      shift_min: int, shift_max: int) -> torch.Tensor:
    """Compact-layout half-spectrum combine (tiled_combine_cuda.py:1142):
    ``dense [n_sb, n_filled_max, t_pad, 2]`` int8 time-minor streams and the
    ``csr`` of ``build_sparse_cell_csr``; writes ONLY the active cells of
    ``out [>= n_fdm, rows, N, N/2+1]`` (complex32, float16 [.., 2] or, here
    also, complex64) at rows ``out_row0 ..``: the caller zeroes the rest.
    ``threads`` and the shift bounds are accepted for the reference's
    signature; this kernel needs neither."""
    n_sb, nfm, t_pad, two = dense.shape
    if two != 2 or n_sb != csr.n_sb:
        raise ValueError(f"dense {tuple(dense.shape)} does not match csr n_sb={csr.n_sb}")
    if dense.dtype != torch.int8 or not dense.is_contiguous():
        raise ValueError("dense must be contiguous int8")
    N = csr.n_grid
    nh = N // 2 + 1
    n_fdm = int(shifts.shape[0])
    if shifts.ndim != 2 or shifts.shape[1] != n_sb:
        raise ValueError(f"shifts must be [n_fdm, n_sb={n_sb}]; got {tuple(shifts.shape)}")
    if not out.is_contiguous():
        raise ValueError("out must be contiguous (pass the parent buffer + out_row0)")
    if out.dtype == torch.complex32:
        tail, f16 = (N, nh), 1
    elif out.dtype == torch.float16:
        tail, f16 = (N, nh, 2), 1
    elif out.dtype == torch.complex64:
        tail, f16 = (N, nh), 0
    else:
        raise ValueError(f"out dtype {out.dtype} not complex32/float16/complex64")
    if int(out.shape[0]) < n_fdm or tuple(out.shape[2:]) != tail:
        raise ValueError(f"out shape {tuple(out.shape)} incompatible with n_fdm={n_fdm} N={N}")
    out_rows = int(out.shape[1])
    if out_row0 < 0 or out_row0 + t_out_len > out_rows:
        raise ValueError(f"out_row0={out_row0} + t_out_len={t_out_len} > rows={out_rows}")
    if t_rows > t_pad:
        raise ValueError(f"t_rows={t_rows} > t_pad={t_pad}")
    for x, nm in ((dense, "dense"), (shifts, "shifts"), (out, "out")):
        _lib.require_cuda(x, nm)
    sh = shifts.to(torch.int32).contiguous()
    st = _lib.status_word(out.device)
    _lib.check(_lib.lib().dsb_combine_sparse(
        _lib.ptr(dense), _lib.ptr(csr.cell_uw), _lib.ptr(csr.cell_ptr), _lib.ptr(csr.ent_g),
        _lib.ptr(csr.ent_k), _lib.ptr(csr.ent_km), csr.n_cells, _lib.ptr(sh), _lib.ptr(out),
        f16, n_sb, int(t_rows), int(t_pad), int(nfm), N, n_fdm, int(t_out_len), int(t_lo),
        int(bool(fftshift)), out_rows, int(out_row0), _lib.ptr(st),
        _lib.stream_of(out.device)), "dsb_combine_sparse")
    _lib.check_status(st, "dsb_combine_sparse")
    return out


# ---------------------------------------------------------------------------
# imaging
# ---------------------------------------------------------------------------


def image_mask_npad(*, n_grid: int, kernel_support: int = 5, sigma_l_pix: Optional[float] = None,
                    envelope_threshold: float = 0.5) -> int:
    """image/imager.py:57-109."""
    if n_grid <= 0 or n_grid & (n_grid - 1):
        raise ValueError(f"n_grid={n_grid}, expected positive power of two")
    if kernel_support < 1:
        raise ValueError(f"kernel_support={kernel_support}, expected ≥ 1")
    if not (0.0 < envelope_threshold <= 1.0):
        raise ValueError(f"envelope_threshold={envelope_threshold}, expected ∈ (0, 1]")
    pad_kernel = (kernel_support // 2) + 2
    pad_env = 0
    if sigma_l_pix is not None and sigma_l_pix > 0:
        rad = float(sigma_l_pix) * math.sqrt(2.0 * math.log(1.0 / envelope_threshold))
        pad_env = max(0, int(math.ceil((n_grid / 2.0) - rad)))
    return max(pad_kernel, pad_env)


def compute_edge_mask(*, n_grid: int, kernel_support: int = 5, sigma_l_pix=None,
                      envelope_threshold: float = 0.5, drop_dc: bool = True,
                      dtype=np.float32, apply_ifft2_dc_correction: bool = True) -> np.ndarray:
    """image/imager.py:112-176 (host table, built once per operating point)."""
    npad = image_mask_npad(n_grid=n_grid, kernel_support=kernel_support,
                           sigma_l_pix=sigma_l_pix, envelope_threshold=envelope_threshold)
    mask = np.zeros((n_grid, n_grid), dtype=dtype)
    if 2 * npad < n_grid:
        mask[npad:n_grid - npad, npad:n_grid - npad] = 1.0
    if drop_dc:
        mask[n_grid // 2, n_grid // 2] = 0.0
    if apply_ifft2_dc_correction:
        ii, jj = np.indices((n_grid, n_grid))
        mask = mask * (1.0 - 2.0 * ((ii + jj) & 1)).astype(dtype)
    return mask


_TWIDDLES: dict = {}


def twiddles(n_grid: int, device) -> torch.Tensor:
    """(N,) complex64 exp(+2 pi i e / N) on ``device`` (cached)."""
    key = (int(n_grid), str(device))
    if key not in _TWIDDLES:
        e = np.arange(n_grid)
        _TWIDDLES[key] = torch.from_numpy(
            np.exp(2j * np.pi * e / n_grid).astype(np.complex64)).to(device)
    return _TWIDDLES[key]


def irfft2_image(half: torch.Tensor, n_grid: int, out: Optional[torch.Tensor] = None
                 ) -> torch.Tensor:
    """Real image from the (fftshift-folded) Hermitian half spectrum
    ``[..., N, N/2+1]`` complex64 -> ``[..., N, N]`` float32: the inverse
    real 2-D FFT of torch.fft.irfft2 (image/imager_gpu.py:590) on this
    library's own kernels (``dsb_irfft2``).  ``half`` is the kernel's work
    buffer: it is overwritten."""
    _lib.require_cuda(half, "half")
    N = int(n_grid)
    if half.dtype != torch.complex64 or tuple(half.shape[-2:]) != (N, N // 2 + 1):
        raise ValueError(f"half must be complex64 [..., {N}, {N // 2 + 1}]")
    if not half.is_contiguous():
        raise ValueError("half must be contiguous")
    lead = tuple(half.shape[:-2])
    n_img = int(np.prod(lead)) if lead else 1
    if out is None:
        out = torch.empty(lead + (N, N), dtype=torch.float32, device=half.device)
    elif out.dtype != torch.float32 or tuple(out.shape) != lead + (N, N) or \
            not out.is_contiguous():
        raise ValueError(f"out must be contiguous float32 {lead + (N, N)}")
    _lib.check(_lib.lib().dsb_irfft2(_lib.ptr(half), n_img, N,
                                     _lib.ptr(twiddles(N, half.device)), _lib.ptr(out),
                                     _lib.stream_of(half.device)), "dsb_irfft2")
    return out


def mask_into_cube(img: torch.Tensor, mask: torch.Tensor, cube: torch.Tensor, f0: int) -> None:
    """``cube[t, f0+f, :, :] = img[f, t] * mask[(f,)]`` (imager_gpu.py:604-650)."""
    _lib.require_cuda(img, "img")
    _lib.require_cuda(cube, "cube")
    n_f, n_t, H, W = img.shape
    per_f = int(mask.ndim == 3)
    _lib.check(_lib.lib().dsb_mask_to_cube(
        _lib.ptr(img), _lib.ptr(mask), per_f, n_f, n_t, H * W, _lib.ptr(cube),
        int(cube.dtype == torch.float16), int(cube.shape[1]), int(f0),
        _lib.stream_of(img.device)), "dsb_mask_to_cube")


@dataclass
class GpuImagerConfig:
    """GPU imager geometry (image/imager_gpu.py:74-117 defaults).  The
    spectrum is complex64 and the transform float32 here (the reference's
    default is complex32); ``cube_dtype`` is the output cube's."""

    n_grid: int = 256
    t_det: int = 256
    n_fdm: int = 32
    n_chgroup: int = 16
    kernel_support: int = 5
    sigma_l_pix: Optional[float] = None
    envelope_threshold: float = 0.5
    drop_dc: bool = True
    cube_dtype: torch.dtype = torch.float16
    complex_dtype: torch.dtype = torch.complex64
    device: Optional[torch.device] = None
    imager_uv_prescale: float = 1.0

    def resolved_device(self) -> torch.device:
        return _lib.cuda_device(self.device if self.device is not None else "cuda")


class GpuImager:
    """Stateful imager for one cube of dense cint8 streams
    (image/imager_gpu.py:123-790): per fine DM the half-spectrum combine
    (``fused_dequant_combine_per_fdm_half``, fftshift folded in), the
    inverse real FFT, and the edge mask (or the per-fine-DM mask of
    ``set_edge_mask_per_fdm``) into ``output_cube [t_det, n_fdm, N, N]``;
    two output cubes alternate, so a returned cube stays valid until the
    next-but-one call.  Combine, transform (``dsb_irfft2``) and mask are this
    library's kernels.  The streaming pipeline itself uses the fused
    ``dsb_image_fft`` path instead."""

    def __init__(self, config: GpuImagerConfig, device: torch.device, edge_mask_real, output_cube,
                 output_cube_alt, uv_slab):
        self.config = config
        self.device = device
        self.edge_mask_real = edge_mask_real
        self.edge_mask_per_fdm: Optional[torch.Tensor] = None
        self.output_cube = output_cube
        self.output_cube_alt = output_cube_alt
        self.uv_slab = uv_slab
        self._flip = False

    @classmethod
    def build(cls, config: GpuImagerConfig) -> "GpuImager":
        """Allocate the persistent buffers and the edge mask (no compute)."""
        if config.complex_dtype != torch.complex64:
            raise ValueError("this imager transforms in float32: complex_dtype must be complex64")
        dev = config.resolved_device()
        N = config.n_grid
        edge = compute_edge_mask(n_grid=N, kernel_support=config.kernel_support,
                                 sigma_l_pix=config.sigma_l_pix,
                                 envelope_threshold=config.envelope_threshold,
                                 drop_dc=config.drop_dc)
        edge_t = torch.from_numpy(edge).to(device=dev, dtype=torch.float32)
        shape = (config.t_det, config.n_fdm, N, N)
        out = torch.empty(shape, dtype=config.cube_dtype, device=dev)
        out_alt = torch.empty(shape, dtype=config.cube_dtype, device=dev)
        uv = torch.empty((config.t_det, N, N // 2 + 1), dtype=torch.complex64, device=dev)
        return cls(config, dev, edge_t, out, out_alt, uv)

    def _img_buffer(self, n_t: int) -> torch.Tensor:
        N = self.config.n_grid
        buf = getattr(self, "_img", None)
        if buf is None or buf.shape[0] < n_t:
            buf = self._img = torch.empty((self.config.t_det, N, N), dtype=torch.float32,
                                          device=self.device)
        return buf[:n_t]

    def set_edge_mask_per_fdm(self, sigma_inv: Optional[torch.Tensor]) -> None:
        """``edge_mask * sigma_inv[f]`` per fine DM (the Layer-1 divide fused
        into the mask), or back to the common mask with None
        (imager_gpu.py:724-790)."""
        if sigma_inv is None:
            self.edge_mask_per_fdm = None
            return
        if sigma_inv.shape != (self.config.n_fdm,):
            raise ValueError(f"sigma_inv.shape={tuple(sigma_inv.shape)}, expected "
                             f"({self.config.n_fdm},)")
        self.edge_mask_per_fdm = (self.edge_mask_real[None, :, :] *
                                  sigma_inv.to(self.device, torch.float32)[:, None, None]
                                  ).contiguous()

    def process_cube(self, *, streams_cint8: torch.Tensor, time_shifts_gpu: torch.Tensor,
                     chgroup_scales: Optional[torch.Tensor] = None,
                     chgroup_offsets_re: Optional[torch.Tensor] = None,
                     chgroup_offsets_im: Optional[torch.Tensor] = None, t_lo: int = 0,
                     compact_inv_lut: Optional[torch.Tensor] = None, compact_t_stream: int = 0,
                     compact_shift_bounds: Optional[tuple] = None) -> torch.Tensor:
        """One cube: ``streams_cint8 [G, T_stream, 2, N, N]`` int8 and
        ``time_shifts_gpu [n_fdm, G]`` int32 -> ``[t_det, n_fdm, N, N]``
        (imager_gpu.py:217-657); with ``compact_inv_lut`` the streams are the
        compact time-minor ``[G, n_filled_max, t_pad, 2]`` and the combine is
        ``combine_sparse_v4``."""
        cfg = self.config
        if time_shifts_gpu.shape != (cfg.n_fdm, streams_cint8.shape[0]):
            raise ValueError(f"time_shifts_gpu shape {tuple(time_shifts_gpu.shape)}, expected "
                             f"({cfg.n_fdm}, {streams_cint8.shape[0]})")
        N = cfg.n_grid
        n_t = cfg.t_det - t_lo
        uv = self.uv_slab[:n_t]
        cube = self.output_cube_alt if self._flip else self.output_cube
        self._flip = not self._flip
        shifts = time_shifts_gpu.to(torch.int32).contiguous()
        if compact_inv_lut is not None:
            return self._process_compact(streams_cint8, shifts, compact_inv_lut,
                                         int(compact_t_stream), t_lo, cube,
                                         (chgroup_scales, chgroup_offsets_re, chgroup_offsets_im))
        for f in range(cfg.n_fdm):
            fused_dequant_combine_per_fdm_half(streams_cint8, shifts[f], uv,
                                               scales=chgroup_scales,
                                               offsets_re=chgroup_offsets_re,
                                               offsets_im=chgroup_offsets_im, t_lo=t_lo,
                                               fftshift=True)
            if cfg.imager_uv_prescale != 1.0:
                uv.mul_(cfg.imager_uv_prescale)
            img = irfft2_image(uv, N, out=self._img_buffer(n_t))[None]   # (1, n_t, N, N)
            mask = (self.edge_mask_real if self.edge_mask_per_fdm is None
                    else self.edge_mask_per_fdm[f:f + 1])
            mask_into_cube(img.contiguous(), mask, cube[t_lo:] if t_lo else cube, f)
        return cube


    def _process_compact(self, streams, shifts, inv_lut, t_stream, t_lo, cube, calib):
        """The compact path of process_cube (imager_gpu.py:300-330, 487-520):
        ``streams [N_chg, n_filled_max, t_pad, 2]`` int8 time-minor, every
        fine DM combined in one launch (combine_sparse_v4) into a zeroed
        half-spectrum buffer, then the transform and mask per fine DM."""
        cfg = self.config
        N = cfg.n_grid
        if streams.ndim != 4 or streams.shape[3] != 2:
            raise ValueError("compact combine expects [N_chg, n_filled_max, t_pad, 2]; "
                             f"got {tuple(streams.shape)}")
        if int(streams.shape[0]) != cfg.n_chgroup:
            raise ValueError(f"compact N_chg={streams.shape[0]} != config "
                             f"N_chgroup={cfg.n_chgroup}")
        if any(x is not None for x in calib):
            raise ValueError("compact combine is the unit-scale path only; per-chgroup "
                             "calibration needs the dense combine")
        if t_stream < cfg.t_det:
            raise ValueError(f"compact_t_stream={t_stream} < T_det={cfg.t_det}")
        key = (int(inv_lut.data_ptr()), tuple(inv_lut.shape), N)
        if getattr(self, "_csr_key", None) != key:
            self._csr = build_sparse_cell_csr(inv_lut, n_grid=N)
            self._csr_key = key
        full = getattr(self, "_uv_full", None)
        if full is None:
            full = self._uv_full = torch.empty((cfg.n_fdm, cfg.t_det, N, N // 2 + 1),
                                               dtype=torch.complex64, device=self.device)
        full[:, t_lo:cfg.t_det].zero_()
        combine_sparse_v4(streams, self._csr, shifts, t_rows=t_stream,
                          t_out_len=cfg.t_det - t_lo, t_lo=t_lo, fftshift=True, out=full,
                          out_row0=t_lo, shift_min=0, shift_max=0)
        n_t = cfg.t_det - t_lo
        for f in range(cfg.n_fdm):
            uv = full[f, t_lo:cfg.t_det]
            if cfg.imager_uv_prescale != 1.0:
                uv.mul_(cfg.imager_uv_prescale)
            img = irfft2_image(uv.contiguous(), N, out=self._img_buffer(n_t))[None]
            mask = (self.edge_mask_real if self.edge_mask_per_fdm is None
                    else self.edge_mask_per_fdm[f:f + 1])
            mask_into_cube(img.contiguous(), mask, cube[t_lo:] if t_lo else cube, f)
        return cube


# ---------------------------------------------------------------------------
# detector
# ---------------------------------------------------------------------------


def precompute_padded_cumsum(x: torch.Tensor, *, axis: int, max_width: int,
                             accum_dtype: Optional[torch.dtype] = None) -> torch.Tensor:
    """Zero-prefixed, max-width-padded float32 cumsum (detector/forward.py:250)."""
    if max_width < 1:
        raise ValueError(f"max_width={max_width}, expected ≥ 1")
    n = x.shape[axis]
    if max_width > n:
        raise ValueError(f"max_width={max_width} exceeds axis-{axis} length {n}")
    if accum_dtype not in (None, torch.float32):
        raise ValueError("dsb200 cumsum is float32 (float64 running prefix)")
    if x.dtype not in (torch.float16, torch.float32):
        raise ValueError(f"x dtype {x.dtype} not supported")
    _lib.require_cuda(x, "x")
    xm = torch.movedim(x, axis, 0).contiguous()
    inner = xm[0].numel()
    cs = torch.empty((n + max_width,) + tuple(xm.shape[1:]), dtype=torch.float32, device=x.device)
    _lib.check(_lib.lib().dsb_padded_cumsum(_lib.ptr(xm), int(xm.dtype == torch.float16), n,
                                            inner, max_width, _lib.ptr(cs),
                                            _lib.stream_of(x.device)), "dsb_padded_cumsum")
    return torch.movedim(cs, 0, axis)


def boxcar_from_padded_cumsum(cs: torch.Tensor, *, axis: int, width: int, max_width: int,
                              n_out: int, t_base: int = 0, out_dtype=None,
                              w_tile_size=None) -> torch.Tensor:
    """Centred boxcar from the padded cumsum (detector/forward.py:339)."""
    if width < 1 or width > max_width:
        raise ValueError(f"width={width} not in [1, max_width={max_width}]")
    if t_base < 0:
        raise ValueError(f"t_base must be >= 0; got {t_base}")
    start = t_base + max_width // 2 - width // 2
    if start + width + n_out > int(cs.shape[axis]):
        raise ValueError("Requested (t_base, n_out, width) window exceeds padded cumsum bounds")
    c = torch.movedim(cs, axis, 0).contiguous()
    _lib.require_cuda(c, "cs")
    out = torch.empty((n_out,) + tuple(c.shape[1:]), dtype=torch.float32, device=c.device)
    _lib.check(_lib.lib().dsb_boxcar_from_cs(_lib.ptr(c), c[0].numel(), width, start, n_out,
                                             _lib.ptr(out), _lib.stream_of(c.device)),
               "dsb_boxcar_from_cs")
    out = torch.movedim(out, 0, axis)
    return out if out_dtype is None else out.to(out_dtype)


def multi_boxcar_argmax_triton(cs: torch.Tensor, *, widths: torch.Tensor, offsets: torch.Tensor,
                               sigma_inv: torch.Tensor, n_out: int, t_base: int = 0,
                               out_max_dtype: Optional[torch.dtype] = None
                               ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Fused multi-width boxcar max + winner (triton_boxcar.py:305).  Same
    name and arguments as the reference (whose Triton kernel this replaces);
    raises instead of returning ``None`` on unsupported inputs."""
    if cs.dim() != 4 or cs.dtype != torch.float32:
        raise ValueError("cs must be float32 [Tpad, F, H, W]")
    _lib.require_cuda(cs, "cs")
    K = int(widths.numel())
    if K < 1 or K > 32 or offsets.numel() != K or sigma_inv.numel() != K:
        raise ValueError("widths/offsets/sigma_inv must have the same length 1..32")
    if widths.dtype != torch.int32 or offsets.dtype != torch.int32 or sigma_inv.dtype != torch.float32:
        raise ValueError("widths/offsets int32, sigma_inv float32")
    eff = out_max_dtype if out_max_dtype is not None else cs.dtype
    if eff not in (torch.float16, torch.float32):
        raise ValueError(f"out_max_dtype {eff} not supported")
    inner = cs[0].numel()
    out_max = torch.empty((n_out,) + tuple(cs.shape[1:]), dtype=eff, device=cs.device)
    out_win = torch.empty((n_out,) + tuple(cs.shape[1:]), dtype=torch.int16, device=cs.device)
    _lib.check(_lib.lib().dsb_multi_boxcar_argmax(
        _lib.ptr(cs), inner, _lib.ptr(widths.contiguous()), _lib.ptr(offsets.contiguous()),
        _lib.ptr(sigma_inv.contiguous()), K, int(n_out), int(t_base), _lib.ptr(out_max),
        int(eff == torch.float16), _lib.ptr(out_win), _lib.stream_of(cs.device)),
        "dsb_multi_boxcar_argmax")
    return out_max, out_win


@dataclass
class Candidate:
    """Detector output (common/contracts.py:256 subset used by the hot path)."""

    l: float
    m: float
    dm_fine: float
    dm_idx: int
    event_specnum: int
    width_samples: int
    kernel_id: str
    snr: float
    flags: int = 0


def _nms(items, *, threshold, n_top, shape, r_t, r_f, r_lm):
    """items: (snr, flat_index, k) with snr > threshold; value-descending then
    flat-index-ascending order, top n_top, greedy merge-radius suppression
    (decoder.py:455-540)."""
    T, F, H, W = shape
    items = sorted(items, key=lambda x: (-x[0], x[1]))[:n_top]
    acc, out = [], []
    for v, ix, k in items:
        if v <= threshold:
            break
        t = ix // (F * H * W)
        rem = ix % (F * H * W)
        f = rem // (H * W)
        rem %= H * W
        l_, m_ = rem // W, rem % W
        if any(abs(t - a) <= r_t and abs(f - b) <= r_f and abs(l_ - c) <= r_lm and abs(m_ - d) <= r_lm
               for a, b, c, d in acc):
            continue
        acc.append((t, f, l_, m_))
        out.append((t, f, l_, m_, v, k))
    return out


def decode_topk_argmax_lowmem(score: torch.Tensor, winner_kernel_idx: torch.Tensor, *,
                              threshold: float, kernel_ids: List[str],
                              kernel_time_widths: List[int], merge_radius_lm: int,
                              merge_radius_fdm: int, merge_radius_t: int,
                              event_specnum: int = 0, fine_to_coarse=None, fine_dm_pc_cm3=None,
                              n_top: int = 256, **_unused) -> List[Candidate]:
    """Top-k + merge-radius decode (decoder.py:388).  Cells above threshold
    are compacted on the device; ties order by flat index ascending."""
    if score.dim() != 4:
        raise ValueError(f"score.dim()={score.dim()}, expected 4 [T_det, N_fdm, H, W]")
    if winner_kernel_idx.shape != score.shape:
        raise ValueError("winner_kernel_idx.shape != score.shape")
    if min(merge_radius_lm, merge_radius_fdm, merge_radius_t) < 0:
        raise ValueError("merge radii must be >= 0")
    if len(kernel_ids) != len(kernel_time_widths):
        raise ValueError("kernel_ids and kernel_time_widths length mismatch")
    if not kernel_ids:
        return []
    flat = score.reshape(-1)
    sel = torch.nonzero(flat > threshold).reshape(-1)
    if sel.numel() == 0:
        return []
    vals = flat[sel].float().cpu().numpy()
    idx = sel.cpu().numpy()
    ks = winner_kernel_idx.reshape(-1)[sel].cpu().numpy()
    got = _nms([(float(v), int(i), int(k)) for v, i, k in zip(vals, idx, ks)], threshold=threshold,
               n_top=n_top, shape=tuple(score.shape), r_t=merge_radius_t, r_f=merge_radius_fdm,
               r_lm=merge_radius_lm)
    f2c = None if fine_to_coarse is None else np.asarray(torch.as_tensor(fine_to_coarse).cpu())
    fdm = None if fine_dm_pc_cm3 is None else np.asarray(torch.as_tensor(fine_dm_pc_cm3).cpu())
    out = []
    for t, f, l_, m_, v, k in got:
        if k < 0 or k >= len(kernel_ids):
            continue
        out.append(Candidate(l=float(l_), m=float(m_),
                             dm_fine=float(fdm[f]) if fdm is not None else float(f),
                             dm_idx=int(f2c[f]) if f2c is not None else int(f),
                             event_specnum=int(event_specnum) + int(t),
                             width_samples=int(kernel_time_widths[k]), kernel_id=kernel_ids[k],
                             snr=float(v)))
    return out


DET_CAND_DTYPE = np.dtype([("t", np.int32), ("pix", np.int32), ("snr", np.float32),
                           ("k", np.int32)])


class CandidateBuffer:
    """Device buffer the fused detector appends above-threshold cells to.
    ``count`` holds the number of cells found (which may pass the capacity)
    and the bits of the largest S/N among those that did not fit."""

    def __init__(self, device, capacity: int = 1 << 20):
        self.device = device
        self.capacity = int(capacity)
        self.buf = torch.empty(self.capacity * 4, dtype=torch.int32, device=device)
        self.count = torch.zeros(2, dtype=torch.int32, device=device)

    def reset(self):
        self.count.zero_()

    # count[1] as the detector leaves it when one of its shared-memory
    # staging copies did not complete within its bounded wait
    TIMEOUT_BITS = 0x7fc00000

    def _check_timeout(self, dropped: int) -> None:
        if dropped == self.TIMEOUT_BITS:
            raise _lib.DsbError("detector: a staging copy wait timed out (DSB_E_TIMEOUT)")

    def fetch(self) -> np.ndarray:
        cnt = self.count.cpu()
        self._check_timeout(int(cnt[1]))
        n = int(cnt[0])
        if n > self.capacity:
            raise _lib.DsbError(f"detector candidate buffer overflow ({n} > {self.capacity})")
        raw = self.buf[: 4 * n].cpu().numpy()
        return raw.view(DET_CAND_DTYPE)

    def fetch_top(self, n_top: int) -> np.ndarray:
        """The entries that can be among the ``n_top`` largest S/N (the only
        ones a top-n_top decode reads): all of them when there are at most
        ``n_top``, else, selected on the device, every entry whose S/N is at
        least the ``n_top``-th largest (ties included, so that the decode's
        flat-index order among equal values still decides).  When cells did
        not fit the buffer, the selection is exact as long as the largest
        S/N among them lies below the selected ones; otherwise DsbError."""
        cnt = self.count.cpu()
        n, dropped = int(cnt[0]), int(cnt[1])
        self._check_timeout(dropped)
        m = min(n, self.capacity)
        rec = self.buf[: 4 * m].view(m, 4)
        if n <= max(n_top, 0) or m == 0:
            return rec.cpu().numpy().reshape(-1).view(DET_CAND_DTYPE)
        snr = rec[:, 2].contiguous().view(torch.float32)
        vk = float(torch.topk(snr, min(n_top, m)).values[-1])
        out = rec[snr >= vk].cpu().numpy().reshape(-1).view(DET_CAND_DTYPE)
        if n > self.capacity and not float(np.int32(dropped).view(np.float32)) < vk:
            raise _lib.DsbError(f"detector candidate buffer overflow ({n} > {self.capacity}) "
                                "reaches the top entries")
        return out


def detect_cube(cube: torch.Tensor, *, log_max_width: int, sigma_inv: torch.Tensor,
                t_base: int, n_out: int, threshold: float, cands: CandidateBuffer,
                pix_offset: int = 0) -> None:
    """Fused padded-cumsum boxcars (widths 1..2**log_max_width), max over
    widths and threshold compaction on a ``[T, F, H, W]`` cube; candidate
    ``pix`` is the flat ``(f, h, w)`` index plus ``pix_offset``."""
    _lib.require_cuda(cube, "cube")
    n = cube.shape[0]
    inner = cube[0].numel()
    _lib.check(_lib.lib().dsb_detect(_lib.ptr(cube), int(cube.dtype == torch.float16), n, 1,
                                     inner, 0, inner, None, 0, None, int(log_max_width),
                                     _lib.ptr(sigma_inv), int(t_base), int(n_out),
                                     float(threshold), _lib.ptr(cands.buf), cands.capacity,
                                     int(pix_offset), _lib.ptr(cands.count),
                                     _lib.stream_of(cube.device)), "dsb_detect")


def detect_images(img: torch.Tensor, mask: torch.Tensor, *, log_max_width: int,
                  sigma_inv: torch.Tensor, t_base: int, n_out: int, threshold: float,
                  cands: CandidateBuffer, pix_offset: int = 0,
                  sigma_f: Optional[torch.Tensor] = None,
                  layer2: Optional["Layer2Samples"] = None) -> None:
    """Detector on FFT output ``img [F, T, H, W]``, each pixel multiplied while
    reading by ``mask`` (``[F, H, W]`` per fine DM, or one ``[H, W]`` for
    all) and divided by ``sigma_f[F]`` (the Layer-1 sigma) when given.  With
    ``layer2`` the detector also writes that object's per-kernel score
    samples of these fine DMs (``pix_offset`` = first fine DM x H x W)."""
    _lib.require_cuda(img, "img")
    _lib.require_cuda(mask, "mask")
    F, T, H, W = img.shape
    npix = H * W
    if mask.numel() not in (npix, F * npix):
        raise ValueError(f"mask has {mask.numel()} cells; expected {npix} or {F * npix}")
    if sigma_f is not None:
        _lib.require_cuda(sigma_f, "sigma_f")
        if sigma_f.numel() != F or sigma_f.dtype != torch.float32:
            raise ValueError("sigma_f must be float32 [F]")
    l2 = (None, None, None, 0) if layer2 is None else (
        layer2.d_off, layer2.d_ent, layer2.samples, layer2.m)
    _lib.check(_lib.lib().dsb_detect_sampled(
        _lib.ptr(img), int(img.dtype == torch.float16), T, F, npix, T * npix, npix,
        _lib.ptr(mask), npix if mask.numel() == F * npix else 0, _lib.ptr(sigma_f),
        int(log_max_width), _lib.ptr(sigma_inv), int(t_base), int(n_out), float(threshold),
        _lib.ptr(cands.buf), cands.capacity, int(pix_offset), _lib.ptr(cands.count),
        _lib.ptr(l2[0]), _lib.ptr(l2[1]), _lib.ptr(l2[2]), int(l2[3]),
        _lib.stream_of(img.device)), "dsb_detect_sampled")


class Layer2Samples:
    """Where the streaming detector samples each kernel's score for the
    Layer-2 noise estimate (detector/forward.py:1425-1470): ``m`` flat
    indices per kernel k over the cube's interior ``[n_out, F, H, W]``,
    drawn by ``torch.randint`` from a generator seeded with k (on the CPU;
    the reference draws on the cube's device), the ones outside the edge
    mask left NaN (layer2.py's ``spatial_active``).  ``samples [K, m]`` is
    filled by the detector, cube by cube."""

    def __init__(self, *, n_kernels: int, m: int, n_out: int, n_fdm: int, npix: int,
                 active: np.ndarray, device):
        if npix % 256:
            raise ValueError("Layer-2 sampling needs H*W a multiple of 256")
        if n_fdm * npix >= 1 << 31:
            raise ValueError("Layer-2 sampling needs F*H*W below 2^31")
        self.m, self.n_kernels = int(m), int(n_kernels)
        fhw = n_fdm * npix
        total = n_out * fhw
        ents = []
        fill = np.full((n_kernels, m), np.nan, np.float32)
        for k in range(n_kernels):
            gen = torch.Generator(device="cpu")
            gen.manual_seed(int(k))
            idx = torch.randint(0, total, (m,), generator=gen).numpy()
            t_in, cell = idx // fhw, idx % fhw
            act = np.asarray(active, bool).reshape(-1)[cell % npix]
            slot = np.arange(m)
            ents.append(np.stack([cell[act], t_in[act], np.full(act.sum(), k), slot[act]], 1))
        ent = np.concatenate(ents).astype(np.int64)
        order = np.lexsort((ent[:, 3], ent[:, 2], ent[:, 1], ent[:, 0]))
        ent = ent[order]
        n_blk = fhw // 256
        off = np.searchsorted(ent[:, 0], np.arange(n_blk + 1) * 256).astype(np.int32)
        self.entries = ent
        self.d_ent = torch.from_numpy(np.ascontiguousarray(ent.astype(np.int32))).to(device)
        self.d_off = torch.from_numpy(off).to(device)
        self.samples = torch.from_numpy(fill).to(device)


# ---------------------------------------------------------------------------
# Layer-1 noise
# ---------------------------------------------------------------------------


def layer1_sigma(img: torch.Tensor, times: torch.Tensor, pix: torch.Tensor, *,
                 n_sigma: float = 3.0, n_iterations: int = 3,
                 out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Layer-1 sigma of each fine DM of ``img [F, T, H, W]`` over the samples
    at ``times x pix`` (int32): sigma_clipped_std_batched of that subsample,
    with values that are not > 0 reported as 1 (the mask divisor)."""
    _lib.require_cuda(img, "img")
    F, T, H, W = img.shape
    if img.dtype != torch.float32:
        raise ValueError("img must be float32")
    for name, t in (("times", times), ("pix", pix)):
        _lib.require_cuda(t, name)
        if t.dtype != torch.int32:
            raise ValueError(f"{name} must be int32")
    if out is None:
        out = torch.empty(F, dtype=torch.float32, device=img.device)
    _lib.check(_lib.lib().dsb_layer1_sigma(_lib.ptr(img), T * H * W, H * W, F, _lib.ptr(times),
                                           times.numel(), _lib.ptr(pix), pix.numel(),
                                           float(n_sigma), int(n_iterations), _lib.ptr(out),
                                           _lib.stream_of(img.device)), "dsb_layer1_sigma")
    return out


def sigma_clipped_std_batched(samples: torch.Tensor, *, n_sigma: float = 3.0,
                              n_iterations: int = 3,
                              out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Row-wise sigma-clipped std, lower median (noise_norm/layer1.py:53);
    into ``out`` (float32 [B]) when given."""
    if samples.dim() != 2:
        raise ValueError(f"samples.dim()={samples.dim()}, expected 2 [B, M]")
    B, M = samples.shape
    _lib.require_cuda(samples, "samples")
    if B == 0 or M == 0:
        return torch.zeros((B,), dtype=torch.float32, device=samples.device)
    s = samples.to(torch.float32).contiguous()
    if out is None:
        out = torch.empty(B, dtype=torch.float32, device=s.device)
    elif out.dtype != torch.float32 or out.numel() != B or not out.is_contiguous():
        raise ValueError(f"out must be contiguous float32 [{B}]")
    _lib.check(_lib.lib().dsb_clipped_std(_lib.ptr(s), B, M, float(n_sigma), int(n_iterations),
                                          _lib.ptr(out), _lib.stream_of(s.device)),
               "dsb_clipped_std")
    return out
