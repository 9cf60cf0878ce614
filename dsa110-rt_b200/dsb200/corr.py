"""Unpack and fast correlator — drop-in for dsa110-rt's
``unpack_int4_split`` (src/dsart/services/slow_corr_kernel.py:220) and
``FastCorrKernel`` (src/dsart/services/corr_fast_kernel.py:290-413).

Geometry is parametric (the reference hard-codes 96 antennas x 384
channels x 2048 packets); defaults equal the reference's.  All compute runs
in ``libdsb200.so``; tensors must live on a CUDA device.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib
from .constants import (BADA_NPOL, LEGACY_FLUFF_SCALE, NANTS, NCHAN_PER_CHGROUP,
                        NPACKETS_PER_BLOCK, NPOL, NTIMES_PER_PACKET, nbase_of)

_DT = {torch.int8: _lib.DT_INT8, torch.float16: _lib.DT_F16, torch.float32: _lib.DT_F32}


def upper_tri_indices(nants: int = NANTS) -> Tuple[np.ndarray, np.ndarray]:
    """``(a_idx, b_idx)`` with ``b <= a``, ``bls = a(a+1)/2 + b``
    (slow_corr_kernel.py:161)."""
    a = np.repeat(np.arange(nants, dtype=np.int64), np.arange(1, nants + 1))
    b = np.concatenate([np.arange(k + 1, dtype=np.int64) for k in range(nants)])
    return a, b


def _raw_to_device(raw, dev: torch.device) -> torch.Tensor:
    if isinstance(raw, torch.Tensor):
        t = raw.reshape(-1)
        if t.dtype != torch.uint8:
            t = t.view(torch.uint8)
        return t.to(dev, non_blocking=True).contiguous()
    if isinstance(raw, (bytes, bytearray, memoryview)):
        arr = np.frombuffer(raw, dtype=np.uint8)
    elif isinstance(raw, np.ndarray):
        arr = raw if raw.dtype == np.uint8 else raw.view(np.uint8)
    else:
        raise TypeError(f"unsupported raw type {type(raw)!r}")
    return torch.from_numpy(np.ascontiguousarray(arr).reshape(-1)).to(dev)


def unpack_int4_split(
    raw,
    *,
    device="cuda",
    scale: float = LEGACY_FLUFF_SCALE,
    out_dtype: torch.dtype = torch.float16,
    npkt: int = NPACKETS_PER_BLOCK,
    nant: int = NANTS,
    nchan: int = NCHAN_PER_CHGROUP,
) -> Tuple[torch.Tensor, torch.Tensor]:
    """Fluff one on-wire page into ``(real, imag)`` in GEMM layout
    ``(nchan, 2t, 2p, npkt, nant)``.  ``out_dtype`` may also be
    ``torch.int8`` (raw integer codes, ``scale`` ignored)."""
    dev = _lib.cuda_device(device)
    if out_dtype not in _DT:
        raise ValueError(f"out_dtype {out_dtype} not in {list(_DT)}")
    expected = npkt * nant * nchan * NTIMES_PER_PACKET * NPOL
    r = _raw_to_device(raw, dev)
    if r.numel() != expected:
        raise ValueError(f"fada raw size {r.numel()} != expected {expected} "
                         f"(= prod{(npkt, nant, nchan, NTIMES_PER_PACKET, NPOL)})")
    shape = (nchan, NTIMES_PER_PACKET, NPOL, npkt, nant)
    re = torch.empty(shape, dtype=out_dtype, device=dev)
    im = torch.empty(shape, dtype=out_dtype, device=dev)
    _lib.check(_lib.lib().dsb_unpack_int4(_lib.ptr(r), npkt, nant, nchan, _DT[out_dtype],
                                          float(scale), _lib.ptr(re), _lib.ptr(im),
                                          _lib.stream_of(dev)), "dsb_unpack_int4")
    return re, im


def apply_cal_split(real_v: torch.Tensor, imag_v: torch.Tensor, cal_real_fine: torch.Tensor,
                    cal_imag_fine: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """Per-(antenna, fine channel, pol) complex gain on split voltages
    (slow_corr_kernel.py:459-528): ``real*g_re - imag*g_im``,
    ``real*g_im + imag*g_re`` on the GEMM layout ``(nchan, 2, 2, npkt,
    nant)``, gains ``(1 or nchan, 1, 2, 1, nant)``; float16 or float32, the
    reference's eager rounding; new output tensors."""
    if real_v.shape != imag_v.shape:
        raise ValueError(f"real_v shape {tuple(real_v.shape)} != imag_v shape "
                         f"{tuple(imag_v.shape)}")
    if real_v.dim() != 5 or real_v.shape[1] != NTIMES_PER_PACKET or real_v.shape[2] != NPOL:
        raise ValueError(f"voltage shape {tuple(real_v.shape)} is not the GEMM layout "
                         f"(nchan, {NTIMES_PER_PACKET}, {NPOL}, npkt, nant)")
    if real_v.dtype != imag_v.dtype:
        raise ValueError(f"real_v dtype {real_v.dtype} != imag_v dtype {imag_v.dtype}")
    if cal_real_fine.dtype != real_v.dtype or cal_imag_fine.dtype != real_v.dtype:
        raise ValueError(f"cal dtypes ({cal_real_fine.dtype}, {cal_imag_fine.dtype}) != "
                         f"voltage dtype {real_v.dtype}")
    if cal_real_fine.device != real_v.device or cal_imag_fine.device != real_v.device:
        raise ValueError(f"cal devices ({cal_real_fine.device}, {cal_imag_fine.device}) != "
                         f"voltage device {real_v.device}")
    if real_v.dtype not in (torch.float16, torch.float32):
        raise ValueError(f"voltage dtype {real_v.dtype}: float16 or float32 expected")
    nchan, nt, npol, npkt, nant = real_v.shape
    gsh = tuple(cal_real_fine.shape)
    if cal_imag_fine.shape != cal_real_fine.shape or gsh not in (
            (1, 1, npol, 1, nant), (nchan, 1, npol, 1, nant)):
        raise ValueError(f"cal shape {gsh}: (1 or {nchan}, 1, {npol}, 1, {nant}) expected")
    dev = _lib.cuda_device(real_v.device)
    args = [t.contiguous() for t in (real_v, imag_v, cal_real_fine, cal_imag_fine)]
    out_re = torch.empty_like(args[0])
    out_im = torch.empty_like(args[0])
    _lib.check(_lib.lib().dsb_cal_apply(
        _lib.ptr(args[0]), _lib.ptr(args[1]), _lib.ptr(args[2]), _lib.ptr(args[3]),
        int(real_v.dtype == torch.float16), nchan, nt, npol, npkt, nant, gsh[0],
        _lib.ptr(out_re), _lib.ptr(out_im), _lib.stream_of(dev)), "dsb_cal_apply")
    return out_re, out_im


def make_cal_broadcast_tensors(gains_fine: np.ndarray, *, device="cuda",
                               dtype: torch.dtype = torch.float16
                               ) -> Tuple[torch.Tensor, torch.Tensor]:
    """``(nant, nchan, npol)`` complex gains -> ``(cal_real, cal_imag)`` of
    shape ``(nchan, 1, npol, 1, nant)`` (slow_corr_kernel.py:531-569): the
    float64 parts converted to ``dtype`` once, then permuted."""
    g = np.asarray(gains_fine)
    if g.ndim != 3 or g.shape[2] != NPOL:
        raise ValueError(f"gains_fine shape {g.shape}, expected (nant, nchan, {NPOL})")
    out = []
    for part in (np.ascontiguousarray(g.real), np.ascontiguousarray(g.imag)):
        t = torch.from_numpy(part).to(device=device, dtype=dtype)
        out.append(t.permute(1, 2, 0).contiguous().unsqueeze(1).unsqueeze(3))
    return out[0], out[1]


def compute_dec_phase(*, chgroup: int, obs_dec_rad: float, antpos_n: np.ndarray,
                      band=None) -> np.ndarray:
    """DEC-only fringe-stop phase per (antenna, channel), complex128
    (cal/cal_loader.py:209-290): exp(-2 pi i f sin(dec - lat) N_a / c),
    cos and sin taken separately, in the reference's order of operations."""
    import math

    from .constants import DSA110_BAND, PHI_LAT_OVRO_RAD, SPEED_OF_LIGHT_M_S
    band = DSA110_BAND if band is None else band
    if not 0 <= chgroup < band.n_chgroup:
        raise ValueError(f"chgroup={chgroup}, expected 0..{band.n_chgroup - 1}")
    n_a = np.asarray(antpos_n)
    if n_a.ndim != 1:
        raise ValueError(f"antpos_n shape {n_a.shape}, expected (nants,)")
    sin_delta = math.sin(obs_dec_rad - PHI_LAT_OVRO_RAD)
    f_hz = band.freq_table()[chgroup].astype(np.float64) * 1.0e9
    arg = (-2.0 * math.pi * sin_delta / SPEED_OF_LIGHT_M_S
           * f_hz[None, :] * n_a.astype(np.float64, copy=False)[:, None])
    return (np.cos(arg) + 1j * np.sin(arg)).astype(np.complex128)


def apply_rfi_mask_to_raw(raw: torch.Tensor, rfi_mask: Optional[torch.Tensor] = None, *,
                          time_chan_mask: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Zero flagged voltages in raw on-wire pages, in place: the RFI
    excision of ``apply_rfi_mask_to_voltages``
    (services/corr_fast_integration.py:1249-1370) moved ahead of the unpack,
    so the correlator never sees a flagged sample (a zero byte is 0 + 0i).

    ``raw``: uint8 ``(G, npkt, nant, nchan, 2, 2)`` (or one page without G)
    on the GPU.  ``rfi_mask``: bool ``(G, nant, nchan, 2)`` (or ``(nant,
    nchan, 2)`` for one page), True == flagged.  ``time_chan_mask``: bool
    ``(G, n_acc, nchan, 2)`` (or 3-D), True == flagged for that accumulation
    of ``npkt / n_acc`` packets on every antenna.  Raises TypeError for a
    non-bool mask and ValueError for a shape mismatch or an ``n_acc`` that
    does not divide the packets, as the reference does."""
    _lib.require_cuda(raw, "raw")
    if raw.dtype != torch.uint8 or raw.dim() not in (5, 6) or raw.shape[-2:] != (2, 2):
        raise ValueError(f"raw must be uint8 (G, npkt, nant, nchan, 2, 2); got "
                         f"{raw.dtype} {tuple(raw.shape)}")
    pages = raw if raw.dim() == 6 else raw.unsqueeze(0)
    G, npkt, nant, nchan = pages.shape[:4]

    def prep(m, name):
        # one flag byte per entry, a leading page axis (added for one page)
        if m is None:
            return None
        if m.dtype != torch.bool:
            raise TypeError(f"{name} must be bool; got {m.dtype}")
        if m.dim() != 3 + (raw.dim() == 6):
            raise ValueError(f"{name} shape {tuple(m.shape)} does not match the pages")
        return m.reshape((G,) + tuple(m.shape[-3:])).to(raw.device, torch.uint8).contiguous()

    m = prep(rfi_mask, "rfi_mask")
    if m is not None and tuple(m.shape) != (G, nant, nchan, 2):
        raise ValueError(f"rfi_mask shape {tuple(rfi_mask.shape)} != (G, NANTS, NCHAN, NPOL) = "
                         f"({G}, {nant}, {nchan}, 2)")
    tm = prep(time_chan_mask, "time_chan_mask")
    n_acc = 0
    if tm is not None:
        n_acc = int(tm.shape[1])
        if tuple(tm.shape[2:]) != (nchan, 2):
            raise ValueError(f"time_chan_mask shape {tuple(time_chan_mask.shape)} != "
                             f"(n_acc, NCHAN, NPOL) = (*, {nchan}, 2)")
        if n_acc <= 0 or npkt % n_acc:
            raise ValueError(f"time_chan_mask has n_acc={n_acc}, which does not divide the "
                             f"packet axis {npkt}")
    _lib.check(_lib.lib().dsb_rfi_zero_fill(_lib.ptr(raw), G, npkt, nant, nchan, _lib.ptr(m),
                                            _lib.ptr(tm), n_acc, _lib.stream_of(raw.device)),
               "dsb_rfi_zero_fill")
    return raw


def validate_fast_voltage_shape(real_v, imag_v, *, t_int_fast_native: int, nants: int = NANTS,
                                nchan: int = NCHAN_PER_CHGROUP, nvolt_pol: int = NPOL
                                ) -> Tuple[int, int]:
    """Same checks and messages as corr_fast_kernel.py:202-284."""
    if real_v.shape != imag_v.shape:
        raise ValueError(f"real_v shape {tuple(real_v.shape)} != imag_v shape {tuple(imag_v.shape)}")
    if real_v.dtype != imag_v.dtype:
        raise ValueError(f"real_v dtype {real_v.dtype} != imag_v dtype {imag_v.dtype}")
    if real_v.ndim != 5:
        raise ValueError(f"voltage tensor must be 5D (nchan, NTIMES_PER_PACKET, nvolt_pol, "
                         f"n_packets_in, nants), got {real_v.ndim}D shape {tuple(real_v.shape)}")
    nch, nt, npol, n_packets_in, na = tuple(real_v.shape)
    if nch != nchan:
        raise ValueError(f"voltage nchan={nch}, expected {nchan}")
    if nt != NTIMES_PER_PACKET:
        raise ValueError(f"voltage NTIMES_PER_PACKET={nt}, expected {NTIMES_PER_PACKET}")
    if npol != nvolt_pol:
        raise ValueError(f"voltage nvolt_pol={npol}, expected {nvolt_pol}")
    if na != nants:
        raise ValueError(f"voltage nants={na}, expected {nants}")
    if n_packets_in <= 0:
        raise ValueError(f"voltage n_packets_in must be > 0, got {n_packets_in}")
    if t_int_fast_native <= 0:
        raise ValueError(f"t_int_fast_native must be > 0, got {t_int_fast_native}")
    if t_int_fast_native % NTIMES_PER_PACKET != 0:
        raise ValueError(f"t_int_fast_native ({t_int_fast_native}) must be a multiple of "
                         f"NTIMES_PER_PACKET ({NTIMES_PER_PACKET}); the GEMM layout has no "
                         f"sub-packet time axis to split on.")
    ppfv = t_int_fast_native // NTIMES_PER_PACKET
    if n_packets_in % ppfv != 0:
        raise ValueError(f"n_packets_in ({n_packets_in}) not a multiple of "
                         f"packets_per_fast_vis ({ppfv} = t_int_fast_native / NTIMES_PER_PACKET); "
                         f"cannot tile the voltage block evenly into fast-vis integrations.")
    return n_packets_in // ppfv, ppfv


@dataclass
class FastCorrKernel:
    """Fast X-engine (corr_fast_kernel.py:290), both entry points on the
    tcgen05 tensor cores.  ``compute_split`` takes the reference's
    GEMM-layout voltages: int8 codes and fp16 voltages (calibrated ones
    included) as kind::f16 with float32 accumulation, as the reference's
    fp16 HMMA correlator (triton_corr_fused.py:135-138), integer codes
    exact; fp32 voltages as kind::tf32.  ``compute_raw`` correlates
    on-wire bytes directly (kind::i8; Stokes-I + channel sum, integer
    exact).  ``check_status`` raises if the last launch's bounded waits
    gave up."""

    device: torch.device
    t_int_fast_native: int = 8
    nants: int = NANTS
    nchan: int = NCHAN_PER_CHGROUP
    nvolt_pol: int = NPOL
    nbada_pol: int = BADA_NPOL
    accum_dtype: torch.dtype = torch.float32
    _nbase: int = field(init=False)

    def __post_init__(self) -> None:
        self.device = _lib.cuda_device(self.device)
        if self.nbada_pol > self.nvolt_pol:
            raise ValueError(f"nbada_pol ({self.nbada_pol}) > nvolt_pol ({self.nvolt_pol})")
        if self.t_int_fast_native % NTIMES_PER_PACKET != 0:
            raise ValueError(f"t_int_fast_native ({self.t_int_fast_native}) must be a multiple "
                             f"of NTIMES_PER_PACKET ({NTIMES_PER_PACKET})")
        if self.t_int_fast_native <= 0:
            raise ValueError(f"t_int_fast_native must be > 0, got {self.t_int_fast_native}")
        if self.nvolt_pol != 2 or self.nbada_pol != 2:
            raise ValueError("dsb200 correlates both parallel hands (nvolt_pol = nbada_pol = 2)")
        self._nbase = nbase_of(self.nants)

    @property
    def nbase(self) -> int:
        return self._nbase

    def check_status(self) -> None:
        st = getattr(self, "_last_status", None)
        if st is not None:
            _lib.check_status(st, "FastCorrKernel")

    def compute_split(self, real_v: torch.Tensor, imag_v: torch.Tensor, *,
                      n_fv_chunk: Optional[int] = None, fuse_stokes_i: bool = False,
                      chan_sum_factor: int = 1) -> torch.Tensor:
        n_fv, _ = validate_fast_voltage_shape(real_v, imag_v,
                                              t_int_fast_native=self.t_int_fast_native,
                                              nants=self.nants, nchan=self.nchan,
                                              nvolt_pol=self.nvolt_pol)
        for t, nm in ((real_v, "real_v"), (imag_v, "imag_v")):
            if t.device != self.device:
                raise ValueError(f"{nm} on {t.device}, kernel on {self.device}")
        if n_fv_chunk is not None and not (1 <= n_fv_chunk <= n_fv):
            raise ValueError(f"n_fv_chunk={n_fv_chunk} must be in [1, n_fv_total={n_fv}]")
        if real_v.dtype not in _DT:
            raise ValueError(f"voltage dtype {real_v.dtype} not supported")
        re = real_v.contiguous()
        im = imag_v.contiguous()
        if fuse_stokes_i:
            if chan_sum_factor < 1 or self.nchan % chan_sum_factor != 0:
                raise ValueError(f"chan_sum_factor={chan_sum_factor} must be ≥ 1 "
                                 f"and divide nchan={self.nchan}")
            out = torch.empty((n_fv, self._nbase, self.nchan // chan_sum_factor),
                              dtype=torch.complex64, device=self.device)
        else:
            out = torch.empty((n_fv, self._nbase, self.nchan, 2), dtype=torch.complex64,
                              device=self.device)
        st = _lib.status_word(self.device)
        _lib.check(_lib.lib().dsb_corr_split(
            _lib.ptr(re), _lib.ptr(im), _DT[re.dtype], self.nchan, re.shape[3], self.nants,
            self.t_int_fast_native, int(bool(fuse_stokes_i)), int(chan_sum_factor),
            _lib.ptr(out), _lib.ptr(st), _lib.stream_of(self.device)), "dsb_corr_split")
        self._last_status = st
        return out

    def compute_raw(self, raw: torch.Tensor, *, chan_sum_factor: int, npkt: Optional[int] = None,
                    out: Optional[torch.Tensor] = None, layout: str = "tbc",
                    max_ctas: int = 0) -> torch.Tensor:
        """Correlate on-wire bytes ``(n_chgroup?, npkt, nant, nchan, 2, 2)``
        (uint8 on the device) on the tensor cores.  ``layout='tbc'`` returns
        ``(n_fv, nbase, nchan/csf)`` per chgroup (the ``compute_split`` fused
        layout); ``'bct'`` returns ``(nbase, nchan/csf, n_fv)`` (time innermost,
        the stage-1 input layout).  A leading chgroup axis is kept when
        ``raw`` has 6 dims."""
        _lib.require_cuda(raw, "raw")
        if raw.dtype != torch.uint8:
            raise TypeError(f"raw must be uint8, got {raw.dtype}")
        page = self.nants * self.nchan * NTIMES_PER_PACKET * NPOL
        n_g = raw.shape[0] if raw.ndim == 6 else 1
        if npkt is None:
            npkt = raw.numel() // (n_g * page)
        if raw.numel() != n_g * npkt * page:
            raise ValueError(f"raw has {raw.numel()} bytes, expected {n_g}x{npkt}x{page}")
        ppfv = self.t_int_fast_native // NTIMES_PER_PACKET
        if npkt % ppfv:
            raise ValueError(f"npkt={npkt} not a multiple of packets_per_fast_vis={ppfv}")
        n_fv = npkt // ppfv
        ceff = self.nchan // chan_sum_factor
        nb = self._nbase
        if layout == "tbc":
            shape = (n_g, n_fv, nb, ceff)
            strides = (n_fv * nb * ceff, nb * ceff, ceff, 1)
            order = 1
        elif layout == "bct":
            shape = (n_g, nb, ceff, n_fv)
            strides = (nb * ceff * n_fv, 1, ceff * n_fv, n_fv)
            order = 0
        else:
            raise ValueError(f"layout {layout!r} not in ('tbc', 'bct')")
        if out is None:
            out = torch.empty(shape, dtype=torch.complex64, device=self.device)
        st = _lib.status_word(self.device)
        _lib.check(_lib.lib().dsb_corr_tc(
            _lib.ptr(raw), npkt * page, n_g, npkt, self.nants, self.nchan,
            self.t_int_fast_native, chan_sum_factor, order, _lib.ptr(out), *strides, max_ctas,
            _lib.ptr(st), _lib.stream_of(self.device)), "dsb_corr_tc")
        self._last_status = st
        return out if raw.ndim == 6 else out[0]


@dataclass
class SlowCorrKernel:
    """Slow correlator product (slow_corr_kernel.py:576-720): one full-block
    integration per (baseline, channel, pol), ``(NBASE, NCHAN, nbada_pol)``
    complex64, stored at ``bls(a, b)`` as ``conj(E_b) E_a`` (F18).  The same
    X-engine as ``FastCorrKernel.compute_split`` with the tile as long as the
    block and the pols kept apart; the block is summed whole, so
    ``half_fac`` (the reference's sub-batching of the packet axis) does not
    change the result.  Integer codes correlate exactly."""

    device: torch.device
    nants: int = NANTS
    nchan: int = NCHAN_PER_CHGROUP
    nvolt_pol: int = NPOL
    nbada_pol: int = BADA_NPOL
    n_time_samples: int = NPACKETS_PER_BLOCK * NTIMES_PER_PACKET
    half_fac: int = 1
    accum_dtype: torch.dtype = torch.float32
    _fast: FastCorrKernel = field(init=False)

    def __post_init__(self) -> None:
        if self.nbada_pol > self.nvolt_pol:
            raise ValueError(f"nbada_pol ({self.nbada_pol}) > nvolt_pol ({self.nvolt_pol})")
        if self.half_fac <= 0 or self.n_time_samples % self.half_fac != 0:
            raise ValueError(f"n_time_samples ({self.n_time_samples}) not divisible by "
                             f"half_fac ({self.half_fac})")
        self._fast = FastCorrKernel(self.device, t_int_fast_native=self.n_time_samples,
                                    nants=self.nants, nchan=self.nchan)
        self.device = self._fast.device

    def compute_split(self, real_v: torch.Tensor, imag_v: torch.Tensor) -> torch.Tensor:
        """Correlate one block of GEMM-layout voltages ``(NCHAN, 2, NPOL,
        n_time_samples / 2, NANTS)`` -> ``(NBASE, NCHAN, nbada_pol)``."""
        want = (self.nchan, NTIMES_PER_PACKET, self.nvolt_pol,
                self.n_time_samples // NTIMES_PER_PACKET, self.nants)
        for name, t in (("real_v", real_v), ("imag_v", imag_v)):
            if t.device != self.device:
                raise ValueError(f"{name} on {t.device}, kernel on {self.device}")
            if tuple(t.shape) != want:
                raise ValueError(f"{name} shape {tuple(t.shape)}, expected {want}")
        if real_v.dtype != imag_v.dtype:
            raise ValueError(f"real_v dtype {real_v.dtype} != imag_v dtype {imag_v.dtype}")
        vis = self._fast.compute_split(real_v, imag_v, fuse_stokes_i=False)
        return vis[0, :, :, : self.nbada_pol]

