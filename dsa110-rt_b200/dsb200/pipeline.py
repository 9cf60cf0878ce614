"""Streaming fast-search pipeline on one B200: the composition of
``process_block`` (services/corr_fast_integration.py:2063: corr phase
:2229 + consume phase :2476) and ``CubePipeline.process``
(services/cube_pipeline.py:2682) with the inter-node UDP corner turn
replaced by device-resident rings.

Data flow per time chunk of ``chunk_tiles`` fast-vis tiles (time is the
absolute fast-vis tile index from the start of the stream):

  raw pages (G, npkt, nant, nchan, 2, 2) uint8
   -> dsb_corr_tc_grid   : unpack + tcgen05 correlator, Stokes I, channel
                           sum, gridded per summed channel into rows Y
                           (ring indexed by tile time)
   -> dsb_stage1_rows    : coarse-DM shift + sum over summed channels,
                           static-sky subtraction; written at t + shift2 into
                           the stage-2 ring D (so the stage-2 FIFO is an index
                           offset)
   -> per fine-DM batch:
      dsb_image_fft      : fine-DM residual shifts, sum over chgroups into the
                           Hermitian half spectrum (fftshift checkerboard) in
                           shared memory, 2-D inverse real FFT -> image
      dsb_clipped_std    : Layer-1 sigma per fine DM (current cube)
      dsb_detect         : edge mask x 1/sigma applied on read, boxcars
                           1..2**log_max_width, max over widths, threshold
                           compaction
   -> host: top-k (value desc, flat index asc) + merge-radius decode

Detector cubes overlap by 2*t_edge so that their interiors tile time.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Iterable, Iterator, List, Optional

import numpy as np
import torch

from . import _lib
from .constants import DSA110_BAND, NATIVE_SAMPLE_US, Band, nbase_of
from .corr import apply_rfi_mask_to_raw
from .dedisp import DMPlan, compute_stage2_shifts, compute_time_shift_search
from .grid import build_pattern, cell_index_map_for, compute_top_of_band_cell_lambda
from .noise import Layer2State
from .search import (CandidateBuffer, Layer2Samples, _nms, compute_edge_mask, detect_images,
                     layer1_sigma, sigma_clipped_std_batched)


def _pow2_at_least(n: int) -> int:
    return 1 << max(0, int(math.ceil(math.log2(max(1, n)))))


@dataclass
class PipelineConfig:
    nant: int = 96
    band: Band = DSA110_BAND
    npkt_block: int = 8192           # packets (2 samples each) per block per chgroup page
    t_int: int = 8                   # native samples per fast-vis tile
    csf: int = 16                    # channels summed per subband
    n_grid: int = 256
    coarse_dm: np.ndarray = field(default_factory=lambda: np.linspace(0.0, 2000.0, 32))
    fine_per_coarse: int = 16
    fine_dm: Optional[np.ndarray] = None
    fine_to_coarse: Optional[np.ndarray] = None
    log_max_width: int = 4           # boxcars 1, 2, 4, ..., 2**log_max_width
    threshold: float = 7.0
    use_sky: bool = True
    sky_window: int = 8
    sky_warmup: int = 8
    chunk_tiles: int = 512
    fdm_batch: int = 8
    # cells decoded per cube (top by S/N, then merge-radius suppression).
    # None: the reference's streaming rule (detector/forward.py:1383-1399,
    # :1607), 64 per kernel scaled by the cube / interior ratio:
    # max(64, ceil(64 (C + 2 t_edge) / C)) x the number of boxcar widths
    n_top: Optional[int] = None
    merge_radius_t: int = 4
    merge_radius_fdm: int = 5
    merge_radius_lm: int = 3
    l1_times: int = 16
    l1_pixels: int = 256
    cand_capacity: int = 1 << 24     # above-threshold cells one cube may hold
    # stage-2 ring element: "c64" (complex64), "bf16" (the BF16 storage form:
    # each part rounded to nearest-even bf16, accumulated in float32 on read)
    # or "cint8" (the reference's cint8 wire form: every (chgroup, coarse DM,
    # time) row quantised with its own amax/127 scale, dequantised on read)
    ring_dtype: str = "c64"
    # coarse DMs per stage-1 block: None picks the largest of 32, 16, 8 whose
    # shared time window fits; a value forces that group
    stage1_dm_group: Optional[int] = None
    # Layer-2 per-kernel noise (noise_norm/layer2.py; the streaming detector,
    # detector/forward.py:1264): each cube's S/N divides the boxcar sums by
    # the previous cube's sigma_k (seeded with sqrt(width)); the cube's own
    # sigma_k estimate (clipped std of layer2_max_samples score samples per
    # kernel, at most 4096) then updates the state.  Off: the fixed
    # 1/sqrt(width).
    layer2: bool = True
    layer2_max_samples: int = 4096
    # calibration on the fast path: complex gain of every antenna in every
    # summed channel, (n_chgroup, nchan // csf, nant) or anything that
    # broadcasts to it ((nant,): one gain per antenna).  The correlator's
    # gridding epilogue multiplies each visibility by g_a conj(g_b), which is
    # what calibrated voltages give (apply_cal_split) when a gain is the same
    # on the summed channels and both pols.  None: uncalibrated (integer
    # exact).
    gains: Optional[np.ndarray] = None
    layer2_tau_s: float = 30.0
    layer2_n_burnin: int = 30

    def __post_init__(self):
        if self.ring_dtype not in RING_FORMATS:
            raise ValueError(f"ring_dtype must be one of {sorted(RING_FORMATS)}, "
                             f"got {self.ring_dtype!r}")
        self.coarse_dm = np.asarray(self.coarse_dm, np.float64)
        if self.fine_dm is None:
            # fine DMs spread evenly around each coarse DM (v2 plan: coarse at the
            # middle of its bucket, constants.py:240-270)
            nc = self.coarse_dm.size
            step = (self.coarse_dm[1] - self.coarse_dm[0]) if nc > 1 else 1.0
            K = self.fine_per_coarse
            off = (np.arange(K) - (K - 1) / 2.0) * (step / K)
            self.fine_dm = (self.coarse_dm[:, None] + off[None, :]).reshape(-1)
            self.fine_dm = np.maximum(self.fine_dm, 0.0)
            self.fine_to_coarse = np.repeat(np.arange(nc), K)
        self.fine_dm = np.asarray(self.fine_dm, np.float64)
        self.fine_to_coarse = np.asarray(self.fine_to_coarse, np.int64)

    @property
    def decoder_n_top(self) -> int:
        if self.n_top is not None:
            return int(self.n_top)
        C, te = self.chunk_tiles, self.t_edge
        return max(64, math.ceil(64 * (C + 2 * te) / C)) * (self.log_max_width + 1)

    @property
    def t_int_us(self) -> float:
        return self.t_int * NATIVE_SAMPLE_US

    @property
    def n_fv_block(self) -> int:
        return self.npkt_block * 2 // self.t_int

    @property
    def ceff(self) -> int:
        return self.band.nchan // self.csf

    @property
    def t_edge(self) -> int:
        return (1 << self.log_max_width) // 2

    @property
    def block_seconds(self) -> float:
        return self.npkt_block * 2 * NATIVE_SAMPLE_US * 1e-6


# element form of the stage-2 ring -> the kernels' format code
RING_FORMATS = {"c64": 0, "bf16": 1, "cint8": 2}


@dataclass
class Tables:
    """Host-built index tables (one-time, FP64 / integer)."""

    cell_lambda: float
    patterns: list
    n_filled: np.ndarray            # (G,)
    yoff: np.ndarray                # (G*ceff,) int32 first Y row of each (chgroup, subband)
    ycnt: np.ndarray
    row_off: np.ndarray             # (n_rows_y + 1) CSR: baselines gridded into each Y row
    row_bls: np.ndarray
    n_rows_y: int
    y_base: np.ndarray              # (G,) first Y row of each chgroup (even)
    pitch: np.ndarray               # (G,) even row pitch between subbands / coarse DMs
    blk_g: np.ndarray               # stage-1 thread blocks: chgroup, first cell
    blk_c0: np.ndarray
    cell_base: np.ndarray           # (G,) first global cell of each chgroup
    shift1: np.ndarray              # (G, ceff, n_coarse) int32
    max_spread: int                 # largest shift1 spread over a stage-1 DM group
    dm_group: int                   # coarse DMs per stage-1 block (32, 16 or 8)
    shift2: np.ndarray              # (G, n_coarse) int32
    d_base: np.ndarray              # (G,) first D row of each chgroup (even)
    n_rows_d: int
    sfine: np.ndarray               # (n_fine, G) int32
    hc_off: np.ndarray              # combine CSR over half cells
    e_g: np.ndarray
    e_cell: np.ndarray
    img: "ImageTables"              # tables of the fused combine + FFT kernel
    twiddles: np.ndarray            # (N,) complex64 exp(+2 pi i e / N)
    mask: np.ndarray                # (N, N) float32


@dataclass
class ImageTables:
    """Tables of dsb_image_fft: the distinct non-zero half cells S, how every
    pattern cell of every chgroup lands on them, and how the kernel's
    threads and column groups split them."""
    n_s: int
    c_meta: np.ndarray      # uint32 s | conj << 16 | g << 17; chgroup runs padded to 64
    cell_base: np.ndarray   # (G + 1) int32
    c2: np.ndarray          # (n_c2, 2) int32: {k | g << 16, s | conj << 16}
    thr_b: np.ndarray       # (threads + 1) int32: S range of each kernel thread
    gmeta: np.ndarray       # (max_entries / epv, threads, epv) entry metadata (see geometry)
    srot: np.ndarray        # (threads,) uint64: 2 bits per entry: packed | parity << 1
    dcols: np.ndarray       # (n_dense,) int32: packed columns with an entry off n' = 0
    dmask: np.ndarray       # (n_dense,) uint64: their occupied n'
    kcols: np.ndarray       # (n_const,) int32: w' | has entries << 16 (constant or zero columns)
    s_mult: int = 1         # most contributions (pattern cells, both targets) to one S entry
    fold: int = 4           # column passes (N = fold * LC)
    meta_bits: int = 16     # 16: w' | n' << 7 | q << 13 | last << 15 (uint16);
    #                         32: w' | n' << 8 | q << 14 | last << 17 | packed << 18 |
    #                             parity << 19 (uint32, rotation bits in the entry)
    # 32-bit form only: the fold's compact tables, which the device buffer of
    # gmeta carries right after gmeta itself (see fold_bytes)
    fold_code: Optional[np.ndarray] = None   # (max_entries / 8, threads) uint32: entry i's
    #                                          nibble q | last << 3 at bits 4 (i % 8)
    thr_slot: Optional[np.ndarray] = None    # (threads + 1) int32: first slot of each thread
    slot_off: Optional[np.ndarray] = None    # (slots, padded to 8) uint16: n' * (N/2 + 2) + w'
    fold_rot: Optional[np.ndarray] = None    # (threads, 4) uint32: entry i's rotation bits
    #                                          packed | parity << 1 at bits 2 (i % 16) of word i / 16

    def gmeta_device_bytes(self) -> np.ndarray:
        """The bytes of the kernel's gmeta buffer: gmeta, then (32-bit form)
        fold_code, thr_slot padded to 16 bytes, fold_rot and slot_off."""
        parts = [np.ascontiguousarray(self.gmeta).view(np.uint8).reshape(-1)]
        if self.fold_code is not None:
            ts = np.zeros(-(-self.thr_slot.size // 4) * 4, np.int32)
            ts[:self.thr_slot.size] = self.thr_slot
            parts += [self.fold_code.view(np.uint8).reshape(-1), ts.view(np.uint8),
                      self.fold_rot.view(np.uint8).reshape(-1), self.slot_off.view(np.uint8)]
        return np.concatenate(parts)


def image_geometry(N: int) -> dict:
    """The image kernel's geometry for grid size N (dsb_image_geometry):
    column passes, threads, S entries per thread, metadata width, and the S
    capacity of the combine's shared arrays."""
    import ctypes
    g = (ctypes.c_int * 5)()
    rc = int(_lib.lib().dsb_image_geometry(N, g))
    if rc:
        raise ValueError(f"dsb_image_fft does not support N={N}")
    return dict(fold=g[0], threads=g[1], max_entries=g[2], meta_bits=g[3], s_capacity=g[4])


def _split_slots(sizes: np.ndarray, n_threads: int, cap: int) -> np.ndarray:
    """Thread boundaries (n_threads + 1) over consecutive slots of the given
    sizes: whole slots per thread, at most ``cap`` entries each, the
    smallest such maximum found by greedy filling."""
    total = int(sizes.sum())
    lo = max(-(-total // n_threads), int(sizes.max()) if sizes.size else 0)
    for m in range(lo, cap + 1):
        b, cur = [0], 0
        for sz in sizes.tolist():
            if cur + sz > m:
                b.append(b[-1] + cur)
                cur = 0
            cur += sz
        b.append(b[-1] + cur)
        if len(b) - 1 <= n_threads:
            b += [total] * (n_threads + 1 - len(b))
            return np.asarray(b, np.int64)
    raise ValueError(f"dsb_image_fft: {total} half cells do not fit {n_threads} threads x "
                     f"{cap} entries")


def build_image_tables(pats, N: int) -> ImageTables:
    """Half-spectrum cell tables for dsb_image_fft.  Pattern cell (u, w) of
    chgroup g adds to half cell (u, w) when w <= N/2 and, conjugated, to its
    mirror ((N-u) % N, (N-w) % N) when that column is <= N/2 (both for
    w = 0 and w = N/2): the Hermitian fold of fused_combine_cuda.py:560-620."""
    geo = image_geometry(N)
    fold, n_thr, cap, mbits = geo["fold"], geo["threads"], geo["max_entries"], geo["meta_bits"]
    LC, NC = N // fold, N // 2
    G = len(pats)
    if G > 63:
        raise ValueError("dsb_image_fft supports at most 63 chgroups")
    us, ws, gs, ks = [], [], [], []
    for g, p in enumerate(pats):
        us.append(p.ix_row.astype(np.int64))
        ws.append(p.ix_col.astype(np.int64))
        gs.append(np.full(p.ix_row.size, g, np.int64))
        ks.append(np.arange(p.ix_row.size, dtype=np.int64))
    u, w, g, k = (np.concatenate(x) for x in (us, ws, gs, ks))
    if k.size and int(k.max()) >= 1 << 16:
        raise ValueError("dsb_image_fft needs fewer than 65536 cells per chgroup")
    direct = w <= N // 2
    um, wm = (N - u) % N, (N - w) % N
    mirror = wm <= N // 2
    # first target: direct if valid, else the mirror (conjugated)
    t1u = np.where(direct, u, um)
    t1w = np.where(direct, w, wm)
    t1c = (~direct).astype(np.int64)
    both = direct & mirror
    t2u, t2w = um[both], wm[both]
    allu = np.concatenate([t1u, t2u])
    allw = np.concatenate([t1w, t2w])
    packed = (allw == N // 2).astype(np.int64)
    wp = np.where(packed == 1, 0, allw)
    key = ((wp * LC + allu % LC) * fold + allu // LC) * 2 + packed
    ukey, inv = np.unique(key, return_inverse=True)
    n_s = int(ukey.size)
    if n_s >= 1 << 16:
        raise ValueError("dsb_image_fft needs fewer than 65536 distinct half cells")
    if n_s > geo["s_capacity"]:
        raise ValueError(f"dsb_image_fft: {n_s} distinct half cells exceed the kernel's "
                         f"{geo['s_capacity']} at N={N}")
    s_pk = ukey & 1
    s_q = (ukey >> 1) % fold
    s_slot = (ukey >> 1) // fold          # w' * LC + n'
    s_wp, s_n = s_slot // LC, s_slot % LC
    s_u = s_n + LC * s_q
    s_w = np.where(s_pk == 1, N // 2, s_wp)
    last = np.ones(n_s, np.int64)
    last[:-1] = (s_slot[1:] != s_slot[:-1]).astype(np.int64)
    # thread ranges: whole slots (a slot's entries are consecutive in S)
    starts = np.flatnonzero(np.r_[True, s_slot[1:] != s_slot[:-1]])
    thr_b = _split_slots(np.diff(np.r_[starts, n_s]), n_thr, cap)
    owner = np.repeat(np.arange(n_thr), np.diff(thr_b))
    idx = np.arange(n_s) - thr_b[owner]
    parity = (s_u + s_w) & 1
    srot = np.zeros(n_thr, np.uint64)
    fold_code = thr_slot = slot_off = fold_rot = None
    if mbits == 16:
        epv = 8
        gmeta = np.zeros((cap // epv, n_thr, epv), np.uint16)
        gmeta[idx // epv, owner, idx % epv] = (s_wp | (s_n << 7) | (s_q << 13) | (last << 15)
                                               ).astype(np.uint16)
        bits = (s_pk | (parity << 1)).astype(np.uint64) << (2 * idx).astype(np.uint64)
        np.bitwise_or.at(srot, owner, bits)
    else:
        epv = 4
        gmeta = np.zeros((cap // epv, n_thr, epv), np.uint32)
        gmeta[idx // epv, owner, idx % epv] = (s_wp | (s_n << 8) | (s_q << 14) | (last << 17) |
                                               (s_pk << 18) | (parity << 19)).astype(np.uint32)
        # the fold's compact form: a nibble per entry (q | last << 3), and the
        # slots in S order with their column-buffer offsets (each thread's
        # slots are consecutive, from thr_slot[t])
        fold_code = np.zeros((cap // 8, n_thr), np.uint32)
        np.bitwise_or.at(fold_code, (idx // 8, owner),
                         ((s_q | (last << 3)) << (4 * (idx % 8))).astype(np.uint32))
        thr_slot = np.searchsorted(starts, thr_b).astype(np.int32)
        offs = s_n[starts] * (NC + 2) + s_wp[starts]
        slot_off = np.zeros(-(-starts.size // 8) * 8, np.uint16)
        slot_off[:starts.size] = offs.astype(np.uint16)
        fold_rot = np.zeros((n_thr, 4), np.uint32)
        np.bitwise_or.at(fold_rot, (owner, idx // 16),
                         ((s_pk | (parity << 1)) << (2 * (idx % 16))).astype(np.uint32))
    # columns: dense (an entry off n' = 0) get the LC-point transform; the
    # rest are constant (every entry at n' = 0) or zero
    occ = np.zeros(NC, np.uint64)
    np.bitwise_or.at(occ, s_wp, np.left_shift(np.uint64(1), s_n.astype(np.uint64)))
    dense = (occ & ~np.uint64(1)) != 0
    dcols = np.flatnonzero(dense).astype(np.int32)
    kc = np.flatnonzero(~dense)
    kcols = (kc | ((occ[kc] != 0).astype(np.int64) << 16)).astype(np.int32)
    n1 = u.size
    # each chgroup's run padded with 0xffffffff to a whole number of 64-entry
    # double chunks (the kernel's warps walk the runs 64 cells at a time)
    nfs = np.asarray([p.ix_row.size for p in pats], np.int64)
    cell_base = np.concatenate([[0], np.cumsum((nfs + 63) // 64 * 64)])
    c_meta = np.full(int(cell_base[-1]), 0xFFFFFFFF, np.uint32)
    c_meta[cell_base[g] + k] = (inv[:n1] | (t1c << 16) | (g << 17)).astype(np.uint32)
    c2 = np.stack([k[both] | (g[both] << 16), inv[n1:] | (1 << 16)], axis=1).astype(np.int32)
    cell_base = cell_base.astype(np.int32)
    return ImageTables(n_s=n_s, c_meta=c_meta, cell_base=cell_base,
                       c2=np.ascontiguousarray(c2.reshape(-1, 2)),
                       thr_b=thr_b.astype(np.int32), gmeta=gmeta, srot=srot, dcols=dcols,
                       dmask=occ[dcols], kcols=kcols,
                       s_mult=int(np.bincount(inv, minlength=n_s).max()), fold=fold,
                       meta_bits=mbits, fold_code=fold_code, thr_slot=thr_slot,
                       slot_off=slot_off, fold_rot=fold_rot)


def build_tables(cfg: PipelineConfig, antpos_e, antpos_n, device, core_mask=None) -> Tables:
    band, G, ceff, N = cfg.band, cfg.band.n_chgroup, cfg.ceff, cfg.n_grid
    nbase = nbase_of(cfg.nant)
    cell = compute_top_of_band_cell_lambda(antpos_e, antpos_n, n_grid=N, band=band,
                                           is_core_baseline_mask=core_mask)
    pats, cims = [], []
    for g in range(G):
        p = build_pattern(antpos_e, antpos_n, chgroup=g, n_grid=N, chan_sum_factor=cfg.csf,
                          cell_lambda=cell, is_core_baseline_mask=core_mask, band=band,
                          device=device)
        pats.append(p)
        cims.append(cell_index_map_for(p, antpos_e, antpos_n, is_core_baseline_mask=core_mask,
                                       device=device))
    n_filled = np.asarray([p.n_filled for p in pats], np.int64)
    # dense rows with an even pitch per chgroup (two cells per 16-byte access):
    # Y row of (g, s, cell) = y_base[g] + s*pitch[g] + cell, D row of
    # (g, coarse DM d, cell) = d_base[g] + d*pitch[g] + cell; the correlator's
    # group (g, s) writes every cell of its chgroup (0 where no baseline lands)
    pitch = (n_filled + 3) // 4 * 4
    y_base = np.concatenate([[0], np.cumsum(pitch * ceff)])
    n_rows_y = int(y_base[-1])
    yoff = np.zeros(G * ceff, np.int64)
    ycnt = np.zeros(G * ceff, np.int64)
    row_cnt = np.zeros(n_rows_y, np.int64)
    row_bls = []
    for g in range(G):
        for s in range(ceff):
            col = cims[g][:, s]
            valid = np.nonzero(col < n_filled[g])[0]
            order = valid[np.argsort(col[valid], kind="stable")]
            r0 = y_base[g] + s * pitch[g]
            yoff[g * ceff + s] = r0
            ycnt[g * ceff + s] = n_filled[g]
            row_cnt[r0:r0 + n_filled[g]] = np.bincount(col[valid], minlength=int(n_filled[g]))
            row_bls.append(order)
    row_off = np.concatenate([[0], np.cumsum(row_cnt)])
    row_bls = np.concatenate(row_bls)
    cell_base = np.concatenate([[0], np.cumsum(n_filled)])
    # stage-1 thread blocks (never straddling a chgroup)
    bs = int(_lib.lib().dsb_stage1_block_size())
    blk_g = np.concatenate([np.full(-(-int(n) // bs), g) for g, n in enumerate(n_filled)])
    blk_c0 = np.concatenate([np.arange(0, int(n), bs) for n in n_filled])
    # shift tables
    plan = DMPlan(dm_pc_cc=cfg.coarse_dm, t_int_fast_us=cfg.t_int_us, chan_sum_factor=cfg.csf,
                  band=band)
    shift1 = plan.delay_bins_all().astype(np.int32)
    # stage-1 DM group: the largest (32, 16, 8 coarse DMs) whose shared time
    # window (the largest spread of one subband's shifts over the group) fits
    # a block's shared memory
    L = _lib.lib()
    s1 = shift1.reshape(G, ceff, -1)
    dg = max_spread = None
    cands = (int(L.dsb_stage1_dm_group()), 16, 8) if cfg.stage1_dm_group is None \
        else (int(cfg.stage1_dm_group),)
    for cand in cands:
        spread = max(int(np.ptp(s1[:, :, k:k + cand], axis=2).max())
                     for k in range(0, s1.shape[2], cand))
        need = int(L.dsb_stage1_smem_bytes(ceff, cand, spread))
        if 0 < need <= 227 * 1024:
            dg, max_spread = cand, spread
            break
    if dg is None:
        raise ValueError("stage 1: the DM plan's shift spread does not fit shared memory even "
                         "with 8 coarse DMs per block; use more coarse DMs over the range")
    shift2 = np.stack([compute_stage2_shifts(chgroup=g, coarse_dm_pc_cm3=cfg.coarse_dm,
                                             t_int_corr_us=cfg.t_int_us,
                                             band=band).shifts_samples for g in range(G)])
    sfine = compute_time_shift_search(coarse_dm_pc_cm3=cfg.coarse_dm, fine_dm_pc_cm3=cfg.fine_dm,
                                      fine_to_coarse=cfg.fine_to_coarse,
                                      t_int_search_us=cfg.t_int_us, merge_coarse_rounding=True,
                                      band=band)
    n_coarse = cfg.coarse_dm.size
    d_base = np.concatenate([[0], np.cumsum(pitch * n_coarse)])
    # combine CSR over half cells (r, c), c in [0, N/2]
    nh = N // 2 + 1
    ent = [[] for _ in range(N * nh)]
    for g, p in enumerate(pats):
        r = p.ix_row.astype(np.int64)
        c = p.ix_col.astype(np.int64)
        for k in range(r.size):
            if c[k] <= N // 2:
                ent[r[k] * nh + c[k]].append((g, k))
            rm, cm = (N - r[k]) % N, (N - c[k]) % N
            if cm <= N // 2:
                ent[rm * nh + cm].append((g, ~k))
    hc_off = np.zeros(N * nh + 1, np.int64)
    hc_off[1:] = np.cumsum([len(x) for x in ent])
    e_g = np.asarray([g for x in ent for g, _ in x], np.int32)
    e_cell = np.asarray([k for x in ent for _, k in x], np.int32)
    img = build_image_tables(pats, N)
    mask = compute_edge_mask(n_grid=N, kernel_support=1)
    e = np.arange(N)
    tw = np.exp(2j * np.pi * e / N).astype(np.complex64)
    return Tables(cell_lambda=cell, patterns=pats, n_filled=n_filled, max_spread=max_spread,
                  dm_group=dg,
                  yoff=yoff.astype(np.int32), ycnt=ycnt.astype(np.int32),
                  row_off=row_off.astype(np.int32), row_bls=row_bls.astype(np.int32),
                  n_rows_y=n_rows_y, y_base=y_base[:-1].astype(np.int32),
                  pitch=pitch.astype(np.int32),
                  blk_g=blk_g.astype(np.int32), blk_c0=blk_c0.astype(np.int32),
                  cell_base=cell_base[:-1].astype(np.int32),
                  shift1=np.ascontiguousarray(shift1), shift2=shift2.astype(np.int32),
                  d_base=d_base[:-1].astype(np.int32), n_rows_d=int(d_base[-1]),
                  sfine=sfine.astype(np.int32), hc_off=hc_off.astype(np.int32), e_g=e_g,
                  e_cell=e_cell, img=img,
                  twiddles=tw, mask=mask.astype(np.float32))


@dataclass
class StreamCandidate:
    t: int          # absolute fast-vis tile (stage-2 / bottom-of-band time)
    fdm: int        # fine-DM index
    l: int          # image row
    m: int          # image column
    snr: float
    width: int      # boxcar width (tiles)


class SearchPipeline:
    """One-GPU streaming fast search with device-resident rings."""

    def __init__(self, cfg: PipelineConfig, antpos_e, antpos_n, device="cuda", core_mask=None):
        self.cfg = cfg
        self.dev = _lib.cuda_device(device)
        self.tab = build_tables(cfg, antpos_e, antpos_n, self.dev, core_mask)
        T = self.tab
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.dev)  # noqa: E731
        self.d_yoff, self.d_ycnt = d(T.yoff), d(T.ycnt)
        self.d_row_off, self.d_row_bls = d(T.row_off), d(T.row_bls)
        self.d_blk_g, self.d_blk_c0 = d(T.blk_g), d(T.blk_c0)
        self.d_ybase, self.d_pitch = d(T.y_base), d(T.pitch)
        it = T.img
        self.d_img_cmeta = d(it.c_meta.view(np.int32))
        self.d_img_cbase, self.d_img_c2 = d(it.cell_base), d(it.c2)
        self.d_img_thrb = d(it.thr_b)
        self.d_img_gmeta = d(it.gmeta_device_bytes().view(np.int16 if it.meta_bits == 16
                                                          else np.int32))
        self.d_img_srot = d(it.srot.view(np.int64))
        self.d_img_dcols, self.d_img_dmask = d(it.dcols), d(it.dmask.view(np.int64))
        self.d_img_kcols = d(it.kcols)
        self.d_tw = d(T.twiddles)
        self.d_shift1, self.d_shift2 = d(T.shift1), d(T.shift2)
        self.d_dbase = d(T.d_base)
        self.d_nfilled = d(T.n_filled.astype(np.int32))
        self.d_sfine, self.d_f2c = d(T.sfine), d(cfg.fine_to_coarse.astype(np.int32))
        self.d_hc_off, self.d_eg, self.d_ecell = d(T.hc_off), d(T.e_g), d(T.e_cell)
        self.d_mask = d(T.mask)
        C = cfg.chunk_tiles
        if cfg.n_fv_block % C:
            raise ValueError("chunk_tiles must divide the block's fast-vis tile count")
        self.max_sh1 = int(T.shift1.max())
        self.depth1 = max(0, math.ceil(self.max_sh1 / C))
        self.L = max(0, -int(T.sfine.min()))
        self.a = math.ceil(self.L / C)
        te = cfg.t_edge
        # warm-up: the first detector cube all of whose times carry data from
        # every chgroup (the stage-2 delay of the top chgroup has elapsed)
        self.jc_first = math.ceil((int(T.shift2.max()) + max(0, int(T.sfine.max())) + 2 * te) / C)
        self.TY = _pow2_at_least((self.depth1 + 1) * C)
        # stage-2 ring: one time-major segment per (chgroup, coarse DM), as deep
        # as its own stage-2 delay needs (a value written at t + shift2 is read
        # by the image kernel up to (a + 1) chunks + 2 t_edge + the largest
        # fine shift later)
        margin = (self.a + 1) * C + 2 * te + max(0, int(T.sfine.max())) + C
        G, n_coarse = T.shift2.shape
        depth = ((T.shift2.astype(np.int64) + margin + 31) // 32 * 32)
        seg_elems = depth * T.pitch.astype(np.int64)[:, None]
        self.seg_base = np.concatenate([[0], np.cumsum(seg_elems.reshape(-1))]).astype(np.int64)
        self.seg_depth = depth.reshape(-1).astype(np.int32)
        self.d_segbase, self.d_segdepth = d(self.seg_base[:-1]), d(self.seg_depth)
        # time-major rings: Y [time & (TY-1)][row]; D segmented as above
        self.Y = torch.zeros((self.TY, T.n_rows_y), dtype=torch.complex64, device=self.dev)
        # D: complex64 elements, one int32 word of bf16 (re low, im high) or
        # one int16 word of int8 (re low, im high) per cell
        self.ring_fmt = RING_FORMATS[cfg.ring_dtype]
        self.ring_bf16 = self.ring_fmt == 1
        self.D = torch.zeros(int(self.seg_base[-1]),
                             dtype=(torch.complex64, torch.int32, torch.int16)[self.ring_fmt],
                             device=self.dev)
        # cint8: the scale of every ring row (one per segment slot), and the
        # chunk's stage-1 rows in complex64 before they are quantised (one
        # segment of C slots per (chgroup, coarse DM), written without delay)
        # bound rows (formats c64, bf16): the largest |part| stage 1 wrote to
        # each (chgroup, coarse DM) in a chunk, one row per chunk kept alive
        # in the ring (reset when its row comes round again); the image
        # kernel sums in fixed point under it
        self.amax_rows = int(-(-int(depth.max()) // C)) + 2
        self.amax = torch.zeros((self.amax_rows, depth.size), dtype=torch.float32,
                                device=self.dev)
        self.sc_base = np.concatenate([[0], np.cumsum(depth.reshape(-1))]).astype(np.int64)
        self.d_scbase = d(self.sc_base[:-1])
        if self.ring_fmt == 2:
            self.scales = torch.ones(int(self.sc_base[-1]), dtype=torch.float32, device=self.dev)
            x_elems = np.broadcast_to(C * T.pitch.astype(np.int64)[:, None], depth.shape)
            x_base = np.concatenate([[0], np.cumsum(x_elems.reshape(-1))]).astype(np.int64)
            self.d_xbase = d(x_base[:-1])
            self.d_xdepth = d(np.full(depth.size, C, np.int32))
            self.d_zero2 = d(np.zeros(depth.size, np.int32))
            self.X = torch.empty(int(x_base[-1]), dtype=torch.complex64, device=self.dev)
        else:
            self.scales = None
        self.sky = (torch.zeros((T.n_rows_d, cfg.sky_window), dtype=torch.complex128,
                                device=self.dev) if cfg.use_sky else None)
        self.sky_count = self.sky_head = self.sky_seen = 0
        self.status = _lib.status_word(self.dev)
        self.d_gains = None
        if cfg.gains is not None:
            gq = np.broadcast_to(np.asarray(cfg.gains, np.complex64),
                                 (cfg.band.n_chgroup, cfg.ceff, cfg.nant))
            self.d_gains = torch.from_numpy(np.ascontiguousarray(gq)).to(self.dev)
        nt_cube = C + 2 * te
        nb = cfg.fdm_batch
        N = cfg.n_grid
        self.img = torch.empty((nb, nt_cube, N, N), dtype=torch.float32, device=self.dev)
        widths = [1 << k for k in range(cfg.log_max_width + 1)]
        self.widths = widths
        self.sinv = d((np.float32(1.0) / np.sqrt(np.asarray(widths, np.float32))).astype(np.float32))
        self.l2 = self.l2_state = None
        if cfg.layer2:
            if not 1 <= cfg.layer2_max_samples <= 4096:
                raise ValueError("layer2_max_samples must be in [1, 4096]")
            self.l2 = Layer2Samples(n_kernels=len(widths), m=cfg.layer2_max_samples, n_out=C,
                                    n_fdm=cfg.fine_dm.size, npix=N * N,
                                    active=T.mask.reshape(-1) != 0, device=self.dev)
            self.l2_state = Layer2State(len(widths), cube_cadence_s=C * cfg.t_int_us * 1e-6,
                                        tau_s=cfg.layer2_tau_s, n_burnin=cfg.layer2_n_burnin,
                                        n_kernel_max_t=1 << cfg.log_max_width, device=self.dev)
            # the analytic unit-noise value seeds the state (forward.py:746-755)
            self.l2_state._s_k.copy_(torch.tensor([math.sqrt(w) for w in widths],
                                                  dtype=torch.float32))
            self.sinv = torch.reciprocal(torch.clamp(self.l2_state.s_k, min=1e-30))
            self.l2_sig = torch.empty(len(widths), dtype=torch.float32, device=self.dev)
        self.cands = CandidateBuffer(self.dev, cfg.cand_capacity)
        self.chunk = 0              # next absolute chunk index to correlate
        self.out: List[StreamCandidate] = []
        self.timing = False          # record CUDA events around each stage when set
        self.events: dict = {}
        self.launches = 0            # dsb200 kernel launches issued
        self.last_d2h_bytes = 0
        self.keep_sigma = False
        self.l1_sigma: List[torch.Tensor] = []
        # Layer-1 subsample positions (interior times x active pixels)
        act = np.nonzero(T.mask.reshape(-1) != 0)[0]
        self.l1_pix = d(act[np.linspace(0, act.size - 1, cfg.l1_pixels).astype(np.int64)]
                        .astype(np.int32))
        self.l1_t = d((te + np.linspace(0, C - 1, cfg.l1_times).astype(np.int64)).astype(np.int32))
        self.l1_sig = torch.empty(cfg.fdm_batch, dtype=torch.float32, device=self.dev)

    # ------------------------------------------------------------------
    class _Mark:
        def __init__(self, pipe, name):
            self.pipe, self.name = pipe, name

        def __enter__(self):
            if self.pipe.timing:
                self.e0 = torch.cuda.Event(enable_timing=True)
                self.e0.record(torch.cuda.current_stream(self.pipe.dev))

        def __exit__(self, *exc):
            if self.pipe.timing:
                e1 = torch.cuda.Event(enable_timing=True)
                e1.record(torch.cuda.current_stream(self.pipe.dev))
                self.pipe.events.setdefault(self.name, []).append((self.e0, e1))
            return False

    def _mark(self, name: str) -> "_Mark":
        return SearchPipeline._Mark(self, name)

    def skip_warmup(self) -> None:
        """Start the stream in steady state: the next block already runs
        stage 1 and the detector on every chunk (rings start at zero), so that
        every block a benchmark times carries the full per-block work."""
        self.chunk = self.jc_first + self.depth1 + self.a
        self.sky_seen = self.cfg.sky_warmup

    def stage_times_ms(self) -> dict:
        """Mean and total device milliseconds per recorded stage."""
        torch.cuda.synchronize(self.dev)
        out = {}
        for k, v in self.events.items():
            ts = [a.elapsed_time(b) for a, b in v]
            out[k] = {"n": len(ts), "total_ms": float(sum(ts)), "mean_ms": float(np.mean(ts))}
        return out

    def _corr(self, raw: torch.Tensor, p0: int, npkt: int) -> None:
        cfg, T = self.cfg, self.tab
        C = cfg.chunk_tiles
        ppfv = cfg.t_int // 2
        row_bytes = cfg.nant * cfg.band.nchan * 4
        page = npkt * row_bytes
        base = raw.data_ptr() + p0 * row_bytes
        with self._mark("corr"):
            _lib.check(_lib.lib().dsb_corr_tc_grid(
                _lib.ctypes.c_void_p(base), page, cfg.band.n_chgroup, C * ppfv, cfg.nant,
                cfg.band.nchan, cfg.t_int, cfg.csf, _lib.ptr(self.d_yoff), _lib.ptr(self.d_ycnt),
                _lib.ptr(self.d_row_off), _lib.ptr(self.d_row_bls), _lib.ptr(self.Y),
                self.tab.n_rows_y, self.chunk * C, self.TY - 1, 0, _lib.ptr(self.d_gains),
                _lib.ptr(self.status), _lib.stream_of(self.dev)), "dsb_corr_tc_grid")
        self.launches += 1

    def _stage1(self, j: int) -> None:
        cfg, T = self.cfg, self.tab
        C = cfg.chunk_tiles
        sub = int(cfg.use_sky and self.sky_count > 0 and self.sky_seen >= cfg.sky_warmup)
        q8 = self.ring_fmt == 2
        # cint8: stage 1 writes the chunk's rows to X (slot t of C, no delay);
        # the quantiser then moves them into the ring at t + shift2
        arow = None
        if not q8:
            arow = self.amax[j % self.amax_rows]
            arow.zero_()
        with self._mark("stage1"):
            _lib.check(_lib.lib().dsb_stage1_rows(
                _lib.ptr(self.Y), T.n_rows_y, self.TY - 1, int(T.blk_g.size),
                _lib.ptr(self.d_blk_g), _lib.ptr(self.d_blk_c0), _lib.ptr(self.d_ybase),
                _lib.ptr(self.d_pitch), _lib.ptr(self.d_shift1),
                _lib.ptr(self.d_zero2 if q8 else self.d_shift2),
                _lib.ptr(self.d_dbase), _lib.ptr(self.d_nfilled),
                _lib.ptr(self.X if q8 else self.D), 0 if q8 else self.ring_fmt,
                _lib.ptr(self.d_xbase if q8 else self.d_segbase),
                _lib.ptr(self.d_xdepth if q8 else self.d_segdepth), _lib.ptr(arow), j * C, C,
                cfg.coarse_dm.size,
                cfg.ceff, T.dm_group, T.max_spread, _lib.ptr(self.sky), cfg.sky_window,
                self.sky_head,
                self.sky_count, sub, _lib.ptr(self.status), _lib.stream_of(self.dev)),
                "dsb_stage1_rows")
            self.launches += 1
            if q8:
                _lib.check(_lib.lib().dsb_ring_encode_cint8(
                    _lib.ptr(self.X), _lib.ptr(self.d_xbase), C, _lib.ptr(self.d_pitch),
                    _lib.ptr(self.d_nfilled), cfg.band.n_chgroup, cfg.coarse_dm.size,
                    _lib.ptr(self.d_shift2), j * C, _lib.ptr(self.D), _lib.ptr(self.d_segbase),
                    _lib.ptr(self.d_segdepth), _lib.ptr(self.scales), _lib.ptr(self.d_scbase),
                    _lib.ptr(self.status), _lib.stream_of(self.dev)), "dsb_ring_encode_cint8")
                self.launches += 1
        if cfg.use_sky:
            self.sky_count = min(self.sky_count + 1, cfg.sky_window)
            self.sky_head = (self.sky_head + 1) % cfg.sky_window
            self.sky_seen += 1

    def image(self, f0: int, n_f: int, t0: int, n_t: int, out: torch.Tensor,
              max_blocks: int = 0) -> None:
        """Fused combine + irfft2 (fftshifted) of fine DMs [f0, f0 + n_f) at
        absolute times [t0, t0 + n_t) from the stage-2 ring into ``out``
        (n_f, n_t, N, N) float32."""
        cfg, T, it = self.cfg, self.tab, self.tab.img
        N = cfg.n_grid
        if out.shape != (n_f, n_t, N, N) or out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError("out must be contiguous float32 (n_f, n_t, N, N)")
        _lib.check(_lib.lib().dsb_image_fft(
            _lib.ptr(self.D), self.ring_fmt, _lib.ptr(self.d_segbase), _lib.ptr(self.d_segdepth),
            _lib.ptr(self.scales), _lib.ptr(self.d_scbase), _lib.ptr(self.amax),
            _lib.ptr(self.d_shift2), cfg.chunk_tiles, self.amax_rows, cfg.coarse_dm.size,
            _lib.ptr(self.d_img_cmeta),
            _lib.ptr(self.d_img_cbase), _lib.ptr(self.d_img_c2), int(it.c2.shape[0]),
            _lib.ptr(self.d_img_thrb), _lib.ptr(self.d_img_gmeta), _lib.ptr(self.d_img_srot),
            it.n_s, it.s_mult, _lib.ptr(self.d_img_dcols), _lib.ptr(self.d_img_dmask), int(it.dcols.size),
            _lib.ptr(self.d_img_kcols), int(it.kcols.size), _lib.ptr(self.d_pitch),
            _lib.ptr(self.d_nfilled), _lib.ptr(self.d_sfine), _lib.ptr(self.d_f2c),
            _lib.ptr(self.d_tw), f0, n_f, cfg.band.n_chgroup, N, t0, n_t, 1, _lib.ptr(out),
            max_blocks, _lib.ptr(self.status), _lib.stream_of(self.dev)), "dsb_image_fft")

    def _search(self, jc: int, collect: bool = True) -> None:
        self._search_device(jc)
        self._search_host(jc, collect)

    def _search_device(self, jc: int) -> None:
        """The detector cube ending with chunk jc on the device: images,
        Layer-1, detector (candidates and Layer-2 samples), the cube's
        per-kernel sigma into ``l2_sig``.  Launches only: no host sync and no
        allocation, so it can be captured in a CUDA graph."""
        cfg = self.cfg
        C, te, N = cfg.chunk_tiles, cfg.t_edge, cfg.n_grid
        t0 = jc * C - 2 * te
        nt = C + 2 * te
        nfine = cfg.fine_dm.size
        self.cands.reset()
        for f0 in range(0, nfine, cfg.fdm_batch):
            nf = min(cfg.fdm_batch, nfine - f0)
            img = self.img[:nf]
            with self._mark("image"):
                self.image(f0, nf, t0, nt, img)
            with self._mark("layer1"):
                sig = layer1_sigma(img, self.l1_t, self.l1_pix, out=self.l1_sig[:nf])
            with self._mark("detect"):
                detect_images(img, self.d_mask, log_max_width=cfg.log_max_width,
                              sigma_inv=self.sinv, t_base=te, n_out=C, threshold=cfg.threshold,
                              cands=self.cands, pix_offset=f0 * N * N, sigma_f=sig,
                              layer2=self.l2)
            self.launches += 3
            if self.keep_sigma:
                self.l1_sigma.append(sig.clone())
        if self.l2 is not None:
            with self._mark("layer2"):
                sigma_clipped_std_batched(self.l2.samples, out=self.l2_sig)
                self.launches += 1

    def _search_host(self, jc: int, collect: bool = True) -> None:
        """The host side of cube jc, after its device work: the Layer-2
        update (this cube's sigma_k folded into the state that divides the
        next cube's boxcars, written into the same divisor buffer) and the
        candidates' read-back and decode."""
        cfg = self.cfg
        C, te, N = cfg.chunk_tiles, cfg.t_edge, cfg.n_grid
        nfine = cfg.fine_dm.size
        if self.l2 is not None:
            s_k, _ = self.l2_state.update_and_query(per_kernel_sigma=self.l2_sig)
            self.sinv.copy_(torch.reciprocal(torch.clamp(s_k, min=1e-30)))
        if collect:
            got = self.cands.fetch_top(cfg.decoder_n_top)
            self.last_d2h_bytes += 8 + got.nbytes
            self._pending = [(float(c["snr"]), int(c["t"]) * (nfine * N * N) + int(c["pix"]),
                              int(c["k"])) for c in got]
            res = _nms(self._pending, threshold=cfg.threshold, n_top=cfg.decoder_n_top,
                       shape=(C, nfine, N, N), r_t=cfg.merge_radius_t, r_f=cfg.merge_radius_fdm,
                       r_lm=cfg.merge_radius_lm)
            t_first = jc * C - te
            for t, f, l_, m_, v, k in res:
                self.out.append(StreamCandidate(t_first + t, f, l_, m_, v, self.widths[k]))
            self._pending = []

    def block_packets(self, raw: torch.Tensor) -> int:
        """Packets per chgroup page of a raw block ``(G, npkt, nant, nchan,
        2, 2)`` uint8; a block may hold any whole number of chunks
        (``chunk_tiles * t_int / 2`` packets each), so streams can deliver
        blocks of uneven length."""
        cfg = self.cfg
        row = cfg.band.n_chgroup * cfg.nant * cfg.band.nchan * 4
        per_chunk = cfg.chunk_tiles * (cfg.t_int // 2)
        if raw.dtype != torch.uint8 or raw.numel() == 0 or raw.numel() % (row * per_chunk):
            raise ValueError("raw must be uint8 (G, npkt, nant, nchan, 2, 2) with npkt a "
                             f"multiple of {per_chunk} packets")
        return raw.numel() // row

    def process_block(self, raw: torch.Tensor, *, collect: bool = True,
                      rfi_mask: Optional[torch.Tensor] = None,
                      time_chan_mask: Optional[torch.Tensor] = None) -> List[StreamCandidate]:
        """Push one block of raw pages ``(G, npkt, nant, nchan, 2, 2)`` uint8
        (device tensor, or host tensor copied here) through the pipeline;
        returns the candidates whose detector cubes completed.  ``npkt`` is
        any whole number of chunks (``npkt_block`` for the fixed-size
        stream).  ``rfi_mask`` ``(G, nant, nchan, 2)`` and ``time_chan_mask``
        ``(G, n_acc, nchan, 2)`` (bool, True == flagged) zero the flagged
        voltages before the correlator (``apply_rfi_mask_to_raw``; a device
        block is changed in place, as the reference's voltages are)."""
        cfg = self.cfg
        npkt = self.block_packets(raw)
        if raw.device.type != "cuda":
            raw = raw.to(self.dev, non_blocking=True)
        raw = raw.contiguous()
        if rfi_mask is not None or time_chan_mask is not None:
            apply_rfi_mask_to_raw(raw, rfi_mask, time_chan_mask=time_chan_mask)
        self.out = []
        self._pending = []
        self.last_d2h_bytes = 0
        C = cfg.chunk_tiles
        ppfv = cfg.t_int // 2
        for ci in range(npkt // (C * ppfv)):
            self._corr(raw, ci * C * ppfv, npkt)
            j = self.chunk - self.depth1
            if j >= 0:
                self._stage1(j)
                jc = j - self.a
                if jc >= self.jc_first:
                    self._search(jc, collect)
            self.chunk += 1
        return self.out

    def device_block(self, raw: torch.Tensor) -> List[int]:
        """The device work of one block ``raw`` (on this pipeline's device):
        every chunk's correlator and stage 1 and the detector cube it
        completes, launches only (see ``_search_device``).  Returns the cubes
        (chunk indices) whose host work ``host_block`` must then do.  At most
        one cube per block: its candidate and Layer-2 buffers are single."""
        npkt = self.block_packets(raw)
        if raw.device != self.dev:
            raise ValueError("device_block needs the block on the pipeline's device")
        cfg = self.cfg
        C, ppfv = cfg.chunk_tiles, cfg.t_int // 2
        cubes = []
        for ci in range(npkt // (C * ppfv)):
            self._corr(raw, ci * C * ppfv, npkt)
            j = self.chunk - self.depth1
            if j >= 0:
                self._stage1(j)
                jc = j - self.a
                if jc >= self.jc_first:
                    if cubes:
                        raise ValueError("device_block: a block may complete one detector "
                                         "cube (chunk_tiles = the block's tiles)")
                    self._search_device(jc)
                    cubes.append(jc)
            self.chunk += 1
        return cubes

    def host_block(self, cubes: List[int], *, collect: bool = True) -> List[StreamCandidate]:
        """The host work of the cubes ``device_block`` returned, once their
        device work has run: Layer-2 update, candidate read-back, decode."""
        self.out = []
        self.last_d2h_bytes = 0
        for jc in cubes:
            self._search_host(jc, collect)
        return self.out

    def process_blocks(self, blocks: Iterable[torch.Tensor], *,
                       collect: bool = True) -> Iterator[List[StreamCandidate]]:
        """Stream blocks held in (pinned) host memory: while block k runs,
        block k+1 is copied to the device on a separate stream into the other
        of two device buffers, so the host-to-device transfer overlaps the
        compute (the block pipelining of corr_fast_integration.py:2593).
        Yields each block's candidates in order."""
        cfg = self.cfg
        shape = (cfg.band.n_chgroup, cfg.npkt_block, cfg.nant, cfg.band.nchan, 2, 2)
        if getattr(self, "_stage", None) is None:
            self._stage = [torch.empty(shape, dtype=torch.uint8, device=self.dev)
                           for _ in range(2)]
            self._copy_stream = torch.cuda.Stream(self.dev)
        compute = torch.cuda.current_stream(self.dev)
        copied = [torch.cuda.Event(), torch.cuda.Event()]
        free = [None, None]
        t_submit = [0.0, 0.0]
        self.block_latency_s: List[float] = []

        def submit(i: int, host: torch.Tensor) -> None:
            if host.dtype != torch.uint8 or host.numel() != self._stage[0].numel():
                raise ValueError("raw must be uint8 (G, npkt, nant, nchan, 2, 2)")
            q = i % 2
            t_submit[q] = time.perf_counter()
            with torch.cuda.stream(self._copy_stream):
                if free[q] is not None:
                    self._copy_stream.wait_event(free[q])   # block i-2 is done with it
                self._stage[q].view(-1).copy_(host.reshape(-1), non_blocking=True)
                copied[q].record(self._copy_stream)

        it = iter(blocks)
        try:
            nxt = next(it)
        except StopIteration:
            return
        submit(0, nxt)
        i = 0
        while nxt is not None:
            try:
                nxt = next(it)
                submit(i + 1, nxt)
            except StopIteration:
                nxt = None
            q = i % 2
            compute.wait_event(copied[q])
            out = self.process_block(self._stage[q], collect=collect)
            free[q] = torch.cuda.Event()
            free[q].record(compute)
            # block-to-candidate latency: handed in -> its candidates on the host
            # (process_block returns after the last chunk's candidate read-back)
            self.block_latency_s.append(time.perf_counter() - t_submit[q])
            yield out
            i += 1

    def ring_values(self, g: int, d: int, times) -> np.ndarray:
        """Stage-2 ring values of chgroup g, coarse DM d at absolute times
        (as stage 1 wrote them, already delayed by shift2): [len(times), nf]."""
        nf = int(self.tab.n_filled[g])
        pitch = int(self.tab.pitch[g])
        gd = g * self.tab.shift2.shape[1] + d
        base, dep = int(self.seg_base[gd]), int(self.seg_depth[gd])
        seg = self.D[base:base + dep * pitch].view(dep, pitch)
        slots = np.asarray(times, np.int64) % dep
        rows = torch.as_tensor(slots, device=self.dev)
        vals = seg[rows, :nf].cpu().numpy()
        if self.ring_fmt == 0:
            return vals
        if self.ring_fmt == 2:
            q = vals.view(np.int8).reshape(len(slots), nf, 2).astype(np.float32)
            sc = self.scales[int(self.sc_base[gd]) + rows].cpu().numpy()[:, None]
            return (sc * q[..., 0] + 1j * (sc * q[..., 1])).astype(np.complex64)
        w = vals.view(np.uint32)
        return ((w << 16).view(np.float32) + 1j * (w & 0xFFFF0000).view(np.float32)
                ).astype(np.complex64)

    def check_status(self) -> None:
        _lib.check_status(self.status, "pipeline")
