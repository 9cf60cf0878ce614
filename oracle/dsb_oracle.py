"""CPU oracle for the dsa110-rt fast search path — TEST INFRASTRUCTURE ONLY.

This module is the checker, not the product.  It restates, in numpy
(int64 / float64 / sequential float32 where the reference's own CPU path
is float32), every stage of dsa110-rt's fast FRB-search hot path:

    4-bit unpack -> X-engine correlator (Stokes-I, channel sum)
    -> sparsity pattern / nearest-cell gridding
    -> stage-1 coarse-DM shift + grid (CSR gather, sliding window)
    -> static-sky mean subtraction
    -> stage-2 per-coarse-DM delay FIFOs
    -> fine-DM combine (full / Hermitian half-spectrum, checkerboard)
    -> dirty image + edge mask
    -> padded cumsum boxcars, multi-boxcar argmax, top-k decode
    -> Layer-1 sigma-clipped std

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its
``cpu_baseline`` leg and ``--impl reference`` arm) may import it, and only
to check or to time the CPU baseline.  The CUDA product path never calls
into this file.

Parity pin: ``tests/golden/*.npz`` hold outputs of the reference itself
(dsa110-rt ``src/dsart``, imported in the build container) on seeded
inputs at its native geometry; ``tests/test_oracle_golden.py`` checks this
module against every one of them.  All reference citations are
``path:line`` inside the dsa110-rt project.

Geometry is parametric (the reference hard-codes 96 antennas and
16 x 384 channels, ``src/dsart/common/constants.py:67-76,200-208``):
``Band`` reproduces the reference exactly for ``REFERENCE_BAND``.
"""

from __future__ import annotations

import math
from collections import deque
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# Constants (src/dsart/common/constants.py:25,163,178)
# ---------------------------------------------------------------------------

NATIVE_SAMPLE_US = 32.768
K_DM_MS_GHZ2_PC = 4.148808
SPEED_OF_LIGHT_M_S = 299_792_458.0
NTIMES_PER_PACKET = 2
NPOL = 2


# ---------------------------------------------------------------------------
# Band / frequency tables (constants.py:133-151; coarse_dm/dm_plan.py:109-150)
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class Band:
    """Channelisation: ``freq(g, c) = f0 - (ch0 + g*nchan + c) * dnu`` GHz.

    Descending in frequency (constants.py:133-144, ``chan_ascending=False``).
    ``REFERENCE_BAND`` reproduces the reference's hard-wired DSA-110 band.
    """

    n_chgroup: int
    nchan: int              # native channels per chgroup
    f0_ghz: float
    dnu_ghz: float
    ch0: int = 0

    def freq_table(self) -> np.ndarray:
        """``(n_chgroup, nchan)`` float64 GHz (constants.py:133 freq_GHz)."""
        g = np.arange(self.n_chgroup, dtype=np.int64)[:, None]
        c = np.arange(self.nchan, dtype=np.int64)[None, :]
        ch_sys = self.ch0 + g * self.nchan + c
        return self.f0_ghz - ch_sys.astype(np.float64) * self.dnu_ghz

    def summed_freq_table(self, csf: int) -> np.ndarray:
        """Band-centre of each ``csf``-channel group (dm_plan.py:128-182)."""
        full = self.freq_table()
        if csf == 1:
            return full
        return full.reshape(self.n_chgroup, self.nchan // csf, csf).mean(axis=2)

    def chgroup_top(self) -> np.ndarray:
        """``NU_CHGROUP_TOP_GHZ`` (constants.py:147): freq(g, 0)."""
        return self.freq_table()[:, 0].copy()

    def bot_proc(self) -> float:
        """``NU_CHGROUP_BOT_GHZ[-1]`` (constants.py:152): freq(G-1, C-1)."""
        return float(self.freq_table()[-1, -1])


REFERENCE_BAND = Band(n_chgroup=16, nchan=384, f0_ghz=1.530,
                      dnu_ghz=0.250 / 8192, ch0=1024)


def delta_tau_us(nu_low: float, nu_high: float, dm: float) -> float:
    """common/dispersion.py:39-66 (same operation order)."""
    ms = K_DM_MS_GHZ2_PC * dm * (1.0 / (nu_low * nu_low) - 1.0 / (nu_high * nu_high))
    return 1000.0 * ms


# ---------------------------------------------------------------------------
# Baseline order (services/slow_corr_kernel.py:161-185)
# ---------------------------------------------------------------------------


def upper_tri_indices(nants: int) -> Tuple[np.ndarray, np.ndarray]:
    """``bls = a(a+1)/2 + b`` with ``b <= a`` (slow_corr_kernel.py:161)."""
    a_idx, b_idx = [], []
    for a in range(nants):
        for b in range(a + 1):
            a_idx.append(a)
            b_idx.append(b)
    return np.asarray(a_idx, np.int64), np.asarray(b_idx, np.int64)


# ---------------------------------------------------------------------------
# a1: int4 unpack (slow_corr_kernel.py:220-405; triton_unpack_onwire.py:51)
# ---------------------------------------------------------------------------


def unpack_nibbles(raw: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Low nibble = real, high nibble = imag, two's complement (int8).

    ``real = ((int8)b << 4) >> 4``, ``imag = (int8)b >> 4``
    (slow_corr_kernel.py:394-396).  Shape preserved.
    """
    b = raw.astype(np.int16)
    lo = b & 0xF
    hi = (b >> 4) & 0xF
    re = np.where(lo >= 8, lo - 16, lo).astype(np.int8)
    im = np.where(hi >= 8, hi - 16, hi).astype(np.int8)
    return re, im


def unpack_int4_gemm_layout(raw: np.ndarray, npkt: int, nant: int, nchan: int
                            ) -> Tuple[np.ndarray, np.ndarray]:
    """On-wire ``(npkt, nant, nchan, 2t, 2p)`` -> GEMM layout
    ``(nchan, 2t, 2p, npkt, nant)`` int8 codes (slow_corr_kernel.py:220;
    the reference additionally multiplies by ``scale``)."""
    r = np.asarray(raw, np.uint8).reshape(npkt, nant, nchan, NTIMES_PER_PACKET, NPOL)
    re, im = unpack_nibbles(r)
    perm = (2, 3, 4, 0, 1)
    return (np.ascontiguousarray(re.transpose(perm)),
            np.ascontiguousarray(im.transpose(perm)))


def rfi_zero_fill_raw(page: np.ndarray, rfi_mask: Optional[np.ndarray],
                      time_chan_mask: Optional[np.ndarray] = None) -> np.ndarray:
    """RFI excision by voltage zero-fill (apply_rfi_mask_to_voltages,
    services/corr_fast_integration.py:1249-1370) applied to one on-wire page
    ``(npkt, nant, nchan, 2t, 2p)`` uint8: every sample of a flagged (antenna,
    channel, pol) of ``rfi_mask (nant, nchan, 2)``, and of a flagged (chan,
    pol) in accumulation a of ``time_chan_mask (n_acc, nchan, 2)`` (packets
    [a * npkt / n_acc, (a + 1) * npkt / n_acc), every antenna), becomes 0:
    both nibbles zero is the voltage 0 + 0i.  True == flagged.  Returns a
    copy."""
    out = np.array(page, np.uint8, copy=True)
    npkt, nant, nchan = out.shape[:3]
    keep = np.ones((npkt, nant, nchan, 1, 2), bool)
    if rfi_mask is not None:
        keep &= ~np.asarray(rfi_mask, bool)[None, :, :, None, :]
    if time_chan_mask is not None:
        tm = np.asarray(time_chan_mask, bool)
        n_acc = tm.shape[0]
        per = npkt // n_acc
        keep &= ~np.repeat(tm, per, axis=0)[:, None, :, None, :]
    out[~np.broadcast_to(keep, out.shape)] = 0
    return out


# ---------------------------------------------------------------------------
# a3: per-antenna complex gains (services/slow_corr_kernel.py:417-569,
# cal/cal_loader.py:209-290)
# ---------------------------------------------------------------------------


def apply_cal_split(re: np.ndarray, im: np.ndarray, g_re: np.ndarray, g_im: np.ndarray
                    ) -> Tuple[np.ndarray, np.ndarray]:
    """``_apply_cal_split_eager`` (slow_corr_kernel.py:417-423) one array op
    at a time in the arrays' dtype: numpy's float16 arithmetic, like torch's,
    computes each op in float32 and rounds the result to half."""
    out_re = re * g_re - im * g_im
    out_im = re * g_im + im * g_re
    return out_re, out_im


def make_cal_broadcast(gains_fine: np.ndarray, dtype=np.float16) -> Tuple[np.ndarray, np.ndarray]:
    """``make_cal_broadcast_tensors`` (slow_corr_kernel.py:531-569): parts
    of ``(nant, nchan, npol)`` gains -> ``(nchan, 1, npol, 1, nant)``."""
    out = []
    for part in (np.ascontiguousarray(gains_fine.real), np.ascontiguousarray(gains_fine.imag)):
        out.append(part.astype(dtype).transpose(1, 2, 0)[:, None, :, None, :].copy())
    return out[0], out[1]


def dec_phase(band: Band, chgroup: int, obs_dec_rad: float, antpos_n: np.ndarray,
              lat_rad: float, c_m_s: float = 299_792_458.0) -> np.ndarray:
    """``compute_dec_phase`` (cal_loader.py:209-290): exp(-2 pi i f sin(dec -
    lat) N_a / c) per (antenna, channel), complex128."""
    import math
    sin_delta = math.sin(obs_dec_rad - lat_rad)
    f_hz = band.freq_table()[chgroup].astype(np.float64) * 1.0e9
    arg = -2.0 * math.pi * sin_delta / c_m_s * f_hz[None, :] * np.asarray(
        antpos_n, np.float64)[:, None]
    return (np.cos(arg) + 1j * np.sin(arg)).astype(np.complex128)


# ---------------------------------------------------------------------------
# a4: fast correlator (services/corr_fast_kernel.py:364-755)
# ---------------------------------------------------------------------------


def corr_fast(re: np.ndarray, im: np.ndarray, *, t_int: int, csf: int = 1,
              fuse_stokes_i: bool = True) -> Tuple[np.ndarray, np.ndarray]:
    """Integer X-engine on GEMM-layout codes ``(nchan, 2t, 2p, npkt, nant)``.

    ``V[b,a] = sum_k conj(E_b) E_a`` over the ``t_int`` native samples of
    each fast-vis tile, stored at ``bls(a, b)`` (F18;
    corr_fast_kernel.py:586-755, triton_corr_fused.py:140-152).
    ``fuse_stokes_i``: sum both pols and ``csf`` channels -> ``(n_fv, nbase,
    nchan // csf)``; else ``(n_fv, nbase, nchan, 2)``.
    Returns ``(vis_re, vis_im)`` int64 (exact).  Implemented with float64
    BLAS matmuls, exact for these integer magnitudes (< 2**53).
    """
    nchan, nt, npol, npkt, nant = re.shape
    ppfv = t_int // NTIMES_PER_PACKET
    n_fv = npkt // ppfv
    a_idx, b_idx = upper_tri_indices(nant)
    nbase = a_idx.size
    if fuse_stokes_i:
        ceff = nchan // csf
        out_re = np.zeros((n_fv, nbase, ceff), np.int64)
        out_im = np.zeros((n_fv, nbase, ceff), np.int64)
    else:
        out_re = np.zeros((n_fv, nbase, nchan, npol), np.int64)
        out_im = np.zeros((n_fv, nbase, nchan, npol), np.int64)
    # (nchan, 2t, 2p, n_fv, ppfv, nant) -> (n_fv, nchan, 2p, 2t*ppfv, nant)
    R = re.astype(np.float64).reshape(nchan, nt, npol, n_fv, ppfv, nant)
    I = im.astype(np.float64).reshape(nchan, nt, npol, n_fv, ppfv, nant)
    R = R.transpose(3, 0, 2, 1, 4, 5).reshape(n_fv, nchan, npol, nt * ppfv, nant)
    I = I.transpose(3, 0, 2, 1, 4, 5).reshape(n_fv, nchan, npol, nt * ppfv, nant)
    if fuse_stokes_i:
        # Stokes I and the channel sum folded into the contraction: the
        # products of a subband's channels and both pols summed by one matmul
        # over K = csf * 2p * 2t * ppfv (exact: integer sums far below 2**53)
        ceff = nchan // csf
        Rk = R.reshape(n_fv, ceff, csf * npol * nt * ppfv, nant)
        Ik = I.reshape(n_fv, ceff, csf * npol * nt * ppfv, nant)
        step = max(1, 4096 // max(1, ceff))
        for f0 in range(0, n_fv, step):
            f1 = min(n_fv, f0 + step)
            r, i = Rk[f0:f1], Ik[f0:f1]
            rt, it = np.swapaxes(r, -1, -2), np.swapaxes(i, -1, -2)
            vre = rt @ r + it @ i            # (f, ceff, nant, nant): [m, n]
            vim = rt @ i - it @ r
            out_re[f0:f1] = np.rint(vre[..., b_idx, a_idx]).astype(np.int64).transpose(0, 2, 1)
            out_im[f0:f1] = np.rint(vim[..., b_idx, a_idx]).astype(np.int64).transpose(0, 2, 1)
        return out_re, out_im
    step = max(1, 64 // max(1, nchan // 16))
    for f0 in range(0, n_fv, step):
        f1 = min(n_fv, f0 + step)
        r = R[f0:f1]
        i = I[f0:f1]
        rt = np.swapaxes(r, -1, -2)
        it = np.swapaxes(i, -1, -2)
        vre = rt @ r + it @ i            # (f, ch, p, nant, nant): [m, n]
        vim = rt @ i - it @ r
        # vis[bls] = V[b, a]  (F18 b/a swap)
        g_re = vre[..., b_idx, a_idx]     # (f, ch, p, nbase)
        g_im = vim[..., b_idx, a_idx]
        g_re = np.rint(g_re).astype(np.int64)
        g_im = np.rint(g_im).astype(np.int64)
        if fuse_stokes_i:
            s_re = g_re.sum(axis=2)       # (f, ch, nbase)
            s_im = g_im.sum(axis=2)
            s_re = s_re.reshape(f1 - f0, nchan // csf, csf, nbase).sum(axis=2)
            s_im = s_im.reshape(f1 - f0, nchan // csf, csf, nbase).sum(axis=2)
            out_re[f0:f1] = s_re.transpose(0, 2, 1)
            out_im[f0:f1] = s_im.transpose(0, 2, 1)
        else:
            out_re[f0:f1] = g_re.transpose(0, 3, 1, 2)
            out_im[f0:f1] = g_im.transpose(0, 3, 1, 2)
    return out_re, out_im


def corr_fast_from_raw(raw: np.ndarray, *, npkt: int, nant: int, nchan: int,
                       t_int: int, csf: int) -> Tuple[np.ndarray, np.ndarray]:
    re, im = unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    return corr_fast(re, im, t_int=t_int, csf=csf, fuse_stokes_i=True)


# ---------------------------------------------------------------------------
# a6: sparsity pattern (grid/sparsity_pattern.py:657-716, 791-860, 893-1198)
# ---------------------------------------------------------------------------


def per_baseline_uv_m(antpos_e, antpos_n, core_mask=None):
    """Kept cross baselines in bls order: ``du = e[a]-e[b]`` (:657-716)."""
    nants = antpos_e.shape[0]
    a_idx, b_idx = upper_tri_indices(nants)
    keep = a_idx != b_idx
    if core_mask is not None:
        keep = keep & np.asarray(core_mask, bool)
    du = antpos_e[a_idx[keep]].astype(np.float64) - antpos_e[b_idx[keep]].astype(np.float64)
    dv = antpos_n[a_idx[keep]].astype(np.float64) - antpos_n[b_idx[keep]].astype(np.float64)
    return du, dv, keep


def top_of_band_cell_lambda(antpos_e, antpos_n, band: Band, n_grid: int,
                            core_mask=None) -> float:
    """F28 common cell scale sized at ``freq(0, 0)`` (:791-860)."""
    du, dv, _ = per_baseline_uv_m(antpos_e, antpos_n, core_mask)
    nu_top = float(band.freq_table()[0, 0])
    wl = SPEED_OF_LIGHT_M_S / (nu_top * 1e9)
    u = du / wl
    v = dv / wl
    return float(np.max(np.maximum(np.abs(u), np.abs(v)))) * 2.0 / n_grid


def uv_cells(antpos_e, antpos_n, band: Band, chgroup: int, csf: int,
             n_grid: int, cell_lambda: float, core_mask=None):
    """Centre cells ``(ix_row, ix_col)`` int64 ``(Nkept, nchan_eff)`` (:1090-1170)."""
    du, dv, keep = per_baseline_uv_m(antpos_e, antpos_n, core_mask)
    nu = band.summed_freq_table(csf)[chgroup]
    wl = SPEED_OF_LIGHT_M_S / (nu * 1e9)
    u = du[:, None] / wl[None, :]
    v = dv[:, None] / wl[None, :]
    u = -u                                   # F20
    v = -v
    half = n_grid // 2
    ix_col = np.rint(u / cell_lambda).astype(np.int64) + half
    ix_row = np.rint(v / cell_lambda).astype(np.int64) + half
    return ix_row, ix_col, keep


def build_pattern(antpos_e, antpos_n, band: Band, chgroup: int, *, n_grid: int,
                  csf: int, cell_lambda: float, core_mask=None):
    """Unique sorted ``(row<<16)|col`` keys of in-grid cells, K=1 (:893-1198)."""
    ix_row, ix_col, _ = uv_cells(antpos_e, antpos_n, band, chgroup, csf,
                                 n_grid, cell_lambda, core_mask)
    ok = (ix_row >= 0) & (ix_row < n_grid) & (ix_col >= 0) & (ix_col < n_grid)
    keys = (ix_row[ok].astype(np.uint32) << 16) | ix_col[ok].astype(np.uint32)
    u = np.unique(keys)
    return ((u >> 16) & 0xFFFF).astype(np.uint16), (u & 0xFFFF).astype(np.uint16)


def cell_index_map(antpos_e, antpos_n, band: Band, chgroup: int, *, n_grid: int,
                   csf: int, cell_lambda: float, ix_row_pat, ix_col_pat,
                   core_mask=None) -> np.ndarray:
    """``(nbase, nchan_eff)`` int64 filled-cell index, sentinel = n_filled
    (grid/kernel.py:308-470, K=1)."""
    nants = antpos_e.shape[0]
    nbase = nants * (nants + 1) // 2
    ix_row, ix_col, keep = uv_cells(antpos_e, antpos_n, band, chgroup, csf,
                                    n_grid, cell_lambda, core_mask)
    n_filled = int(ix_row_pat.size)
    pat_keys = (ix_row_pat.astype(np.uint32) << 16) | ix_col_pat.astype(np.uint32)
    ok = (ix_row >= 0) & (ix_row < n_grid) & (ix_col >= 0) & (ix_col < n_grid)
    keys = (np.where(ok, ix_row, 0).astype(np.uint32) << 16) | np.where(ok, ix_col, 0).astype(np.uint32)
    pos = np.searchsorted(pat_keys, keys)
    pos = np.where(ok, pos, n_filled)
    cim = np.full((nbase, ix_row.shape[1]), n_filled, np.int64)
    cim[np.where(keep)[0]] = pos
    return cim


def grid_vis(vis: np.ndarray, cim: np.ndarray, n_filled: int) -> np.ndarray:
    """``FastVisGridder.compute`` (grid/kernel.py:508-611), K=1: scatter-add
    ``(n_fv, nbase, nchan_eff)`` into ``(n_fv, n_filled)``."""
    n_fv = vis.shape[0]
    flat_idx = cim.reshape(-1)
    out = np.zeros((n_fv, n_filled + 1), dtype=vis.dtype)
    src = vis.reshape(n_fv, -1)
    for f in range(n_fv):
        np.add.at(out[f], flat_idx, src[f])
    return out[:, :n_filled]


# ---------------------------------------------------------------------------
# a8/a19: DM plan delays (coarse_dm/dm_plan.py:194-243, 454-462)
# ---------------------------------------------------------------------------


def delay_native_table(coarse_dm: np.ndarray, freqs: np.ndarray) -> np.ndarray:
    """``(G, C, K)`` int64, Convention A (reference = chgroup top) (:194-243)."""
    nu = freqs.astype(np.float64)
    nu_top = nu[:, 0:1]
    inv_diff = (1.0 / (nu ** 2)) - (1.0 / (nu_top ** 2))
    delay_us = (K_DM_MS_GHZ2_PC * coarse_dm.astype(np.float64)[None, None, :]
                * inv_diff[:, :, None] * 1e3)
    return np.rint(delay_us / NATIVE_SAMPLE_US).astype(np.int64)


def delay_bins(nat: np.ndarray, t_int_fast_us: float) -> np.ndarray:
    """Second rint to fast-vis bins (dm_plan.py:412-462)."""
    t_int_fast_native = float(t_int_fast_us) / NATIVE_SAMPLE_US
    return np.rint(nat / t_int_fast_native).astype(np.int64)


def stage1_bin_shifts(band: Band, coarse_dm, csf: int, t_int_fast_us: float) -> np.ndarray:
    """``(G, C_eff, K)`` stage-1 bin shifts (DMPlan.from_summed_canonical +
    delay_bins_per_chgroup, dm_plan.py:637-697,454-462)."""
    nat = delay_native_table(np.asarray(coarse_dm, np.float64), band.summed_freq_table(csf))
    return delay_bins(nat, t_int_fast_us)


# ---------------------------------------------------------------------------
# a8: stage-1 shift + grid (corr_fast_integration.py:647-700, 917-1046;
#     triton_dedisp.py:50-168)
# ---------------------------------------------------------------------------


def build_cell_csr(cim: np.ndarray, n_filled: int):
    """Per-cell source list ``(offs, b, c)``; sources ordered by flat
    ``b*C + c`` inside each cell (triton_dedisp.py:50-100)."""
    nb, nc = cim.shape
    flat = cim.reshape(-1)
    valid = np.where(flat < n_filled)[0]
    order = valid[np.argsort(flat[valid], kind="stable")]
    counts = np.bincount(flat[valid], minlength=n_filled)
    offs = np.zeros(n_filled + 1, np.int64)
    offs[1:] = np.cumsum(counts)
    return offs, (order // nc).astype(np.int64), (order % nc).astype(np.int64)


def stage1_dedisp(vis: np.ndarray, shifts: np.ndarray, cim: np.ndarray,
                  n_filled: int, t_dedisp: int) -> np.ndarray:
    """``out[d, t, cell] = sum_{(b,c) in cell} vis[t + shift[c, d], b, c]``
    (corr_fast_integration.py:647-700).  ``vis`` ``(T, nbase, C)`` integers
    (or any exact type); ``shifts`` ``(C, n_dm)``.  The sum is taken as the
    reference's gather over each cell's (baseline, channel) sources, grouped
    by channel: first every channel's baselines are summed into its cells,
    then each DM adds the channels' rows at their shifted times.  For integer
    input the result is exact, so the grouping cannot change it."""
    from scipy.sparse import csr_matrix
    T, nb, nc = vis.shape
    n_dm = shifts.shape[1]
    out = np.zeros((n_dm, t_dedisp, n_filled), dtype=vis.dtype)
    b, c = np.nonzero(cim < n_filled)
    if b.size == 0:
        return out
    cell = cim[b, c].astype(np.int64)
    M = csr_matrix((np.ones(b.size, vis.dtype), (b * nc + c, c * n_filled + cell)),
                   shape=(nb * nc, nc * n_filled))
    Y = np.asarray(vis.reshape(T, nb * nc) @ M).reshape(T, nc, n_filled)
    for d in range(n_dm):
        for ch in range(nc):
            sh = int(shifts[ch, d])
            out[d] += Y[sh:sh + t_dedisp, ch]
    return out


class Stage1Window:
    """Sliding-window stage 1 (F34, corr_fast_integration.py:917-1046),
    generalised to ``depth`` blocks of history: the block pushed at call
    ``k`` is emitted at call ``k + depth`` once every shifted read is
    available.  ``depth == 1`` is exactly the reference's F34 (first call
    emits zeros, then the previous block)."""

    def __init__(self, shifts: np.ndarray, cim: np.ndarray, n_filled: int,
                 depth: int = 1):
        self.shifts = shifts
        self.cim = cim
        self.n_filled = n_filled
        self.depth = depth
        self.hist: List[np.ndarray] = []

    def push(self, vis: np.ndarray) -> np.ndarray:
        n_fv = vis.shape[0]
        n_dm = self.shifts.shape[1]
        self.hist.append(vis)
        if len(self.hist) <= self.depth:
            return np.zeros((n_dm, n_fv, self.n_filled), vis.dtype)
        self.hist = self.hist[-(self.depth + 1):]
        joined = np.concatenate(self.hist, axis=0)
        maxs = int(self.shifts.max()) if self.shifts.size else 0
        if joined.shape[0] - maxs < n_fv:
            raise ValueError("history too short for plan max shift")
        return stage1_dedisp(joined, self.shifts, self.cim, self.n_filled, n_fv)


# ---------------------------------------------------------------------------
# a9: static-sky mean (corr_fast_integration.py:1049-1240)
# ---------------------------------------------------------------------------


class StaticSkyMean:
    """Per (DM slot, cell) boxcar mean of the past ``window`` cubes'
    per-cell time means, subtracted from each new cube after ``warmup``
    cubes (:1049-1240).  Oracle state is float64; the cube mean is the
    exact float64 mean of the float32 values and the output is
    ``float32(x - mean)`` (one rounding), the same definition the CUDA
    kernel implements (the reference itself uses complex64 torch ops, so
    its last-ulp rounding is not reproducible from numpy)."""

    def __init__(self, window_blocks: int = 8, warmup_cubes: int = 8, n_dm: int = 1):
        self.window = window_blocks
        self.warmup = warmup_cubes
        self.n_dm = n_dm
        self.ring = [None] * n_dm
        self.count = [0] * n_dm
        self.head = [0] * n_dm
        self.seen = [0] * n_dm

    def apply(self, gridded: np.ndarray, dm_slot: int = 0) -> np.ndarray:
        g = gridded.astype(np.complex128)
        mean = g.mean(axis=0)
        s = dm_slot
        if self.ring[s] is None:
            self.ring[s] = np.zeros((self.window, g.shape[1]), np.complex128)
        if self.count[s] == 0 or self.seen[s] < self.warmup:
            out = gridded.copy()
        else:
            win = self.ring[s][: self.count[s]].sum(axis=0) if self.count[s] < self.window \
                else self.ring[s].sum(axis=0)
            m = win / self.count[s]
            out = (g - m[None, :]).astype(np.complex64)
        self.ring[s][self.head[s]] = mean
        if self.count[s] < self.window:
            self.count[s] += 1
        self.head[s] = (self.head[s] + 1) % self.window
        self.seen[s] += 1
        return out


# ---------------------------------------------------------------------------
# a10: stage-2 shifts and FIFOs (coarse_dm/stage2_shifts.py:170-321;
#      stage2_chgroup_alignment.py:79-338; stage2_per_dm_fifo.py:108-263;
#      stage2_fifo.py:83-291)
# ---------------------------------------------------------------------------


def stage2_shifts(band: Band, chgroup: int, coarse_dm, t_int_corr_us: float) -> np.ndarray:
    """``rint(dtau(nu_bot_proc, nu_top[g], dm_c) / t_int)`` int32 (:170-321)."""
    nu_bot = band.bot_proc()
    nu_g = float(band.chgroup_top()[chgroup])
    dms = np.asarray(coarse_dm, np.float64)
    out = np.zeros(dms.size, np.int32)
    for c in range(dms.size):
        out[c] = int(np.rint(delta_tau_us(nu_bot, nu_g, float(dms[c])) / t_int_corr_us))
    return out


class Stage2InterChgroupShiftFifo:
    """Per-coarse-DM time roll by ``shift[c]`` samples with whole-cube
    warm-up gating (stage2_chgroup_alignment.py:79-338)."""

    def __init__(self, shifts: np.ndarray, t_dedisp: int):
        self.shifts = np.asarray(shifts, np.int64)
        self.T = int(t_dedisp)
        self.k = self.shifts // self.T
        self.r = self.shifts - self.k * self.T
        self.rings = [deque(maxlen=int(self.k[c]) + 2) for c in range(self.shifts.size)]

    def _req(self, c):
        return int(self.k[c]) + 1 if int(self.r[c]) == 0 else int(self.k[c]) + 2

    def push(self, cube: np.ndarray) -> list:
        n_dm = self.shifts.size
        for c in range(n_dm):
            self.rings[c].appendleft(cube[c].copy())
        if not any(len(self.rings[c]) >= self._req(c) for c in range(n_dm)):
            return []
        out = np.zeros_like(cube)
        T = self.T
        for c in range(n_dm):
            if len(self.rings[c]) < self._req(c):
                continue
            k, r = int(self.k[c]), int(self.r[c])
            ring = self.rings[c]
            if r == 0:
                out[c] = ring[k]
            else:
                out[c, 0:r] = ring[k + 1][T - r:T]
                out[c, r:T] = ring[k][0:T - r]
        return [out]


class PerCoarseDmStage2FIFO:
    """Depth ``D`` per coarse DM: push i emits push i-D; ``D == 0`` is a
    pass-through (stage2_per_dm_fifo.py:181-263; tests/test_stage2_per_dm_fifo.py:28-50)."""

    def __init__(self, depths: Sequence[int]):
        self.depths = [int(d) for d in depths]
        self.bufs = [deque() if d > 0 else None for d in self.depths]

    def push(self, c: int, x):
        d = self.depths[c]
        buf = self.bufs[c]
        if d == 0 or buf is None:
            return x
        if len(buf) < d:
            buf.append(x)
            return None
        out = buf.popleft()
        buf.append(x)
        return out


# ---------------------------------------------------------------------------
# a11: fine-DM shift table (fine_dm/combiner.py:150-498)
# ---------------------------------------------------------------------------


def time_shift_search(band: Band, coarse_dm, fine_dm, fine_to_coarse,
                      t_int_us: float, merge_coarse_rounding: bool = True) -> np.ndarray:
    """Signed int32 ``(N_fine, G)`` residual shifts, TOP reference
    (combiner.py:150-498).  Merged rounding (production flag,
    configs/dsart_search_rt.yaml:298): ``rint(dtau(fine)/T) - rint(dtau(coarse)/T)``."""
    tops = band.chgroup_top()
    nu_bot = band.bot_proc()
    coarse_dm = np.asarray(coarse_dm, np.float64)
    fine_dm = np.asarray(fine_dm, np.float64)
    n_fine = fine_dm.size
    G = tops.size
    out = np.zeros((n_fine, G), np.int32)
    for f in range(n_fine):
        c = int(fine_to_coarse[f])
        for g in range(G):
            if merge_coarse_rounding:
                s_f = np.rint(delta_tau_us(nu_bot, float(tops[g]), float(fine_dm[f])) / t_int_us)
                s_c = np.rint(delta_tau_us(nu_bot, float(tops[g]), float(coarse_dm[c])) / t_int_us)
                out[f, g] = int(s_f - s_c)
            else:
                ddm = float(fine_dm[f] - coarse_dm[c])
                out[f, g] = int(np.rint(delta_tau_us(nu_bot, float(tops[g]), ddm) / t_int_us))
    return out


# ---------------------------------------------------------------------------
# a12: fine-DM combine (fine_dm/combiner.py:548-655;
#      image/fused_combine_cuda.py:210-300, 560-620)
# ---------------------------------------------------------------------------


def combine_full(streams: np.ndarray, shifts: np.ndarray, t_det: int, t_lo: int = 0,
                 fftshift: bool = True) -> np.ndarray:
    """``G[t,u,w] = sum_g streams[g, t - shift[g], u, w]`` (zero outside
    ``[0, T_stream)``), checkerboard ``(-1)^(u+w)`` if ``fftshift``."""
    G, Ts, N, _ = streams.shape
    out = np.zeros((t_det - t_lo, N, N), np.complex128)
    for t in range(t_lo, t_det):
        for g in range(G):
            ts = t - int(shifts[g])
            if 0 <= ts < Ts:
                out[t - t_lo] += streams[g, ts]
    if fftshift:
        u = np.arange(N)
        out *= (1 - 2 * ((u[:, None] + u[None, :]) & 1))
    return out


def combine_half(streams: np.ndarray, shifts: np.ndarray, t_det: int, t_lo: int = 0,
                 fftshift: bool = True) -> np.ndarray:
    """Hermitian half-spectrum ``0.5 (G[u,w] + conj G[-u,-w])``, ``w <= N/2``
    (fused_combine_cuda.py:560-620)."""
    return half_from_full(combine_full(streams, shifts, t_det, t_lo, fftshift=False), fftshift)


def half_from_full(full: np.ndarray, fftshift: bool = True) -> np.ndarray:
    """The Hermitian half spectrum of combined grids ``full`` (T, N, N):
    ``0.5 (G[u,w] + conj G[-u,-w])`` for ``w <= N/2``, times the checkerboard
    ``(-1)^(u+w)`` when ``fftshift`` (fused_combine_cuda.py:560-620)."""
    N = full.shape[-1]
    u = np.arange(N)
    # G[-u, -w] for w in [0, N/2]: rows reversed and rolled by one (row 0
    # stays), then column 0 followed by columns N-1 down to N/2
    rows = np.roll(full[:, ::-1, :], 1, axis=1)
    mir = np.concatenate([rows[:, :, :1], rows[:, :, N - 1:N // 2 - 1:-1]], axis=2)
    h = 0.5 * (full[:, :, : N // 2 + 1] + np.conj(mir))
    if fftshift:
        w = np.arange(N // 2 + 1)
        h *= (1 - 2 * ((u[:, None] + w[None, :]) & 1))
    return h


def combine_sparse(dense: np.ndarray, inv_lut: np.ndarray, shifts: np.ndarray, *,
                   t_rows: int, t_out_len: int, t_lo: int = 0,
                   fftshift: bool = True) -> np.ndarray:
    """The compact-layout combine (image/tiled_combine_cuda.py:966-1060):
    ``dense [n_sb, n_filled_max, t_pad, 2]`` int8 time-minor streams,
    ``inv_lut [n_sb, N*N]`` the compact index of each grid cell per stream
    (-1 absent), ``shifts [n_fdm, n_sb]``.  Each stream is scattered back to
    its dense grid and combined as ``combine_half`` does (stream time
    t + t_lo - shift, zero outside [0, t_rows)); returns complex128
    ``[n_fdm, t_out_len, N, N/2+1]`` (exact: the sums are of integers)."""
    n_sb, nfm, t_pad, _ = dense.shape
    N = int(round(np.sqrt(inv_lut.shape[1])))
    streams = np.zeros((n_sb, t_rows, N * N), np.complex128)
    for g in range(n_sb):
        cells = np.flatnonzero(inv_lut[g] >= 0)
        k = inv_lut[g, cells]
        v = dense[g, k, :t_rows].astype(np.float64)            # (cells, t, 2)
        streams[g][:, cells] = (v[..., 0] + 1j * v[..., 1]).T
    streams = streams.reshape(n_sb, t_rows, N, N)
    return np.stack([combine_half(streams, shifts[f], t_lo + t_out_len, t_lo, fftshift=fftshift)
                     for f in range(shifts.shape[0])])


def _fma32(a, b, c):
    """float32 fma: a*b + c rounded once (a*b is exact in float64 for the
    float32 x int8 products used here, and so is the sum at these ranges)."""
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64)
            + np.asarray(c, np.float64)).astype(np.float32)


def combine_dequant(q: np.ndarray, shifts: np.ndarray, scales, off_re, off_im, t_det: int,
                    t_lo: int = 0, half: bool = False, fftshift: bool = True) -> np.ndarray:
    """Calibrated cint8 combine (fused_combine_cuda.py:431-505, :681): each
    chgroup term adds ``fma(scale, q, acc) + offset`` in float32, scale and
    offsets per chgroup ``[G]`` or per (chgroup, source time) ``[G, T]``;
    the half form sums the mirror term the same way and takes
    ``0.5 (direct + conj mirror)``.  ``q``: int8 ``[G, T, 2, N, N]``."""
    G, Ts, _, N, _ = q.shape
    per_t = np.ndim(scales) == 2
    nw = N // 2 + 1 if half else N
    u = np.arange(N)[:, None]
    w = np.arange(nw)[None, :]
    um, wm = (N - u) % N, (N - w) % N
    out = np.zeros((t_det - t_lo, N, nw), np.complex64)
    for t in range(t_lo, t_det):
        ar = np.zeros((N, nw), np.float32)
        ai = np.zeros_like(ar)
        mr = np.zeros_like(ar)
        mi = np.zeros_like(ar)
        for g in range(G):
            ts = t - int(shifts[g])
            if not 0 <= ts < Ts:
                continue
            idx = (g, ts) if per_t else (g,)
            sc = np.float32(np.asarray(scales)[idx])
            orr = np.float32(np.asarray(off_re)[idx])
            oii = np.float32(np.asarray(off_im)[idx])
            re, im = q[g, ts, 0].astype(np.float32), q[g, ts, 1].astype(np.float32)
            ar = (_fma32(sc, re[u, w], ar) + orr).astype(np.float32)
            ai = (_fma32(sc, im[u, w], ai) + oii).astype(np.float32)
            if half:
                mr = (_fma32(sc, re[um, wm], mr) + orr).astype(np.float32)
                mi = (_fma32(sc, im[um, wm], mi) + oii).astype(np.float32)
        if half:
            o_re = (np.float32(0.5) * (ar + mr)).astype(np.float32)
            o_im = (np.float32(0.5) * (ai - mi)).astype(np.float32)
        else:
            o_re, o_im = ar, ai
        if fftshift:
            flip = ((u + w) & 1).astype(bool)
            o_re = np.where(flip, -o_re, o_re)
            o_im = np.where(flip, -o_im, o_im)
        out[t - t_lo] = o_re + 1j * o_im
    return out


# ---------------------------------------------------------------------------
# wire encoding of dedispersed rows (transport/tx.py:803-873)
# ---------------------------------------------------------------------------


def encode_rows(row: np.ndarray, bits_per_cell: int):
    """``TransportTx._encode_rows`` (tx.py:825-873): one DM row ``(n_fv,
    n_filled)`` complex encoded tile by tile.  16 bits per cell: cint8 with
    scale = float32(float64(amax) / 127) over |re|, |im| (1 for an all-zero
    tile) and q = clip(round-half-even(x * float32(1 / scale)), -128, 127);
    32 bits: float16 parts, scale 1.  Returns ``(payloads (n_fv, n_filled,
    2), scales (n_fv,) float32)``."""
    arr = np.asarray(row).astype(np.complex64, copy=False)
    n_fv, n_filled = arr.shape
    re_im = np.empty((n_fv, n_filled, 2), np.float32)
    re_im[:, :, 0] = arr.real
    re_im[:, :, 1] = arr.imag
    if bits_per_cell == 16:
        amax = (np.abs(re_im).reshape(n_fv, -1).max(axis=1) if n_filled
                else np.zeros(n_fv, np.float32))
        scales = (amax.astype(np.float64) / 127.0).astype(np.float32)
        scales[amax == 0.0] = np.float32(1.0)
        inv = (1.0 / scales.astype(np.float64)).astype(np.float32)
        q = np.clip(np.round(re_im * inv[:, None, None]), -128.0, 127.0).astype(np.int8)
        return q, scales
    if bits_per_cell == 32:
        return re_im.astype(np.float16), np.ones(n_fv, np.float32)
    raise AssertionError(f"unhandled bits_per_cell={bits_per_cell}")


def decode_cint8(q: np.ndarray, scales: np.ndarray) -> np.ndarray:
    """Receiver side of the cint8 form: ``(n_fv, n_filled, 2)`` int8 payload
    and ``(n_fv,)`` scales -> complex64 rows, each part float32(scale * q)
    (the per-tile dequantisation of image/fused_combine_cuda.py:431-505)."""
    sc = np.asarray(scales, np.float32)[:, None]
    qf = np.asarray(q).astype(np.float32)
    return (sc * qf[..., 0] + 1j * (sc * qf[..., 1])).astype(np.complex64)


def compact_to_dense(values: np.ndarray, ix_row, ix_col, n_grid: int) -> np.ndarray:
    """Scatter ``(..., n_filled)`` cell values into ``(..., N, N)``."""
    out = np.zeros(values.shape[:-1] + (n_grid, n_grid), values.dtype)
    out[..., ix_row.astype(np.int64), ix_col.astype(np.int64)] = values
    return out


# ---------------------------------------------------------------------------
# a13/a14: imaging (image/imager.py:57-310; image/imager_gpu.py:520-660)
# ---------------------------------------------------------------------------


def image_mask_npad(n_grid: int, kernel_support: int = 5) -> int:
    """imager.py:57-109 with no envelope term."""
    return (kernel_support // 2) + 2


def edge_mask(n_grid: int, kernel_support: int = 5, drop_dc: bool = True,
              dc_correction: bool = True) -> np.ndarray:
    """imager.py:112-176."""
    npad = image_mask_npad(n_grid, kernel_support)
    m = np.zeros((n_grid, n_grid), np.float32)
    if 2 * npad < n_grid:
        m[npad:n_grid - npad, npad:n_grid - npad] = 1.0
    if drop_dc:
        m[n_grid // 2, n_grid // 2] = 0.0
    if dc_correction:
        ii, jj = np.indices((n_grid, n_grid))
        m = m * (1.0 - 2.0 * ((ii + jj) & 1)).astype(np.float32)
    return m


def dirty_image(uv: np.ndarray) -> np.ndarray:
    """``Re(fftshift(ifft2(G)))`` in float64 (imager.py:232-246)."""
    img = np.fft.ifft2(uv, axes=(-2, -1))
    img = np.fft.fftshift(img, axes=(-2, -1))
    return np.real(img)


def image_from_half(half: np.ndarray, n_grid: int) -> np.ndarray:
    """``irfft2`` of the (fftshift-folded) half spectrum (imager_gpu.py:590)."""
    return np.fft.irfft2(half, s=(n_grid, n_grid), axes=(-2, -1))


# ---------------------------------------------------------------------------
# a15/a16: boxcar detector (detector/forward.py:250-455;
#          detector/triton_boxcar.py:193-360)
# ---------------------------------------------------------------------------


def padded_cumsum(x: np.ndarray, max_width: int) -> np.ndarray:
    """Zero-prefixed float32 cumsum along axis 0 with ``max_w//2`` left pad
    and ``max_w-1-max_w//2`` right pad holding the last value (forward.py:250-337).
    Each prefix is accumulated sequentially in float64 and rounded once to
    float32 — what ``torch.cumsum(..., dtype=float32)`` does on the CPU
    (its float accumulator type is double)."""
    n = x.shape[0]
    pl = max_width // 2
    pr = max_width - 1 - pl
    cs = np.zeros((n + max_width,) + x.shape[1:], np.float32)
    cs[1 + pl: 1 + pl + n] = np.cumsum(x.astype(np.float32).astype(np.float64),
                                       axis=0).astype(np.float32)
    if pr > 0:
        cs[1 + pl + n:] = cs[pl + n]
    return cs


def boxcar_offsets(widths: Sequence[int], max_width: int) -> np.ndarray:
    return np.asarray([max_width // 2 - w // 2 for w in widths], np.int64)


def multi_boxcar_argmax(cs: np.ndarray, widths, offsets, sigma_inv, n_out: int,
                        t_base: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """``snr_k = (cs[t+off_k+w_k] - cs[t+off_k]) * sigma_inv_k`` in float32;
    max with strict ``>`` so the lowest k wins ties (triton_boxcar.py:193-290)."""
    t = np.arange(n_out) + t_base
    best = None
    win = None
    for k, (w, off, si) in enumerate(zip(widths, offsets, sigma_inv)):
        hi = cs[t + off + w]
        lo = cs[t + off]
        snr = ((hi - lo).astype(np.float32) * np.float32(si)).astype(np.float32)
        if best is None:
            best = snr
            win = np.zeros(snr.shape, np.int16)
        else:
            better = snr > best
            best = np.where(better, snr, best)
            win = np.where(better, np.int16(k), win)
    return best, win


@dataclass
class Cand:
    t: int
    f: int
    l: int
    m: int
    snr: float
    k: int


def decode_topk(score: np.ndarray, winner: np.ndarray, *, threshold: float, n_top: int,
                r_t: int, r_f: int, r_lm: int) -> List[Cand]:
    """Global top-``n_top`` on ``[T, F, H, W]`` then greedy merge-radius NMS
    (decoder.py:388-540).  Tie order (unspecified for ``torch.topk``) is
    defined here: value descending, then flat index ascending."""
    flat = score.reshape(-1).astype(np.float32)
    if flat.size == 0 or float(flat.max()) <= threshold:
        return []
    idx = np.nonzero(flat > threshold)[0]
    vals = flat[idx]
    order = np.lexsort((idx, -vals.astype(np.float64)))
    idx = idx[order][:n_top]
    T, F, H, W = score.shape
    out: List[Cand] = []
    acc: List[Tuple[int, int, int, int]] = []
    wflat = winner.reshape(-1)
    for ix in idx:
        v = float(flat[ix])
        t = int(ix) // (F * H * W)
        rem = int(ix) % (F * H * W)
        f = rem // (H * W)
        rem = rem % (H * W)
        l_ = rem // W
        m_ = rem % W
        if any(abs(t - at) <= r_t and abs(f - af) <= r_f and abs(l_ - al) <= r_lm
               and abs(m_ - am) <= r_lm for at, af, al, am in acc):
            continue
        acc.append((t, f, l_, m_))
        out.append(Cand(t, f, l_, m_, v, int(wflat[ix])))
    return out


# ---------------------------------------------------------------------------
# a18: Layer-1 sigma-clipped std (noise_norm/layer1.py:53-125)
# ---------------------------------------------------------------------------


def _lower_nanmedian(x: np.ndarray) -> float:
    v = np.sort(x[np.isfinite(x)])
    if v.size == 0:
        return float("nan")
    return float(v[(v.size - 1) // 2])


def sigma_clipped_std_batched(samples: np.ndarray, n_sigma: float = 3.0,
                              n_iterations: int = 3) -> np.ndarray:
    """Row-wise clipped std with torch.nanmedian's LOWER median (layer1.py:53)."""
    s = samples.astype(np.float32)
    out = np.zeros(s.shape[0], np.float32)
    for r in range(s.shape[0]):
        row = s[r]
        active = np.isfinite(row)
        med = np.float32(_lower_nanmedian(np.where(active, row, np.nan)))
        cnt = max(1, int(active.sum()))
        d = np.where(active, row - med, 0).astype(np.float32)
        sig = np.float32(np.sqrt(np.float32(np.sum(d * d, dtype=np.float64)) / np.float32(cnt)))
        for _ in range(n_iterations):
            lo = med - np.float32(n_sigma) * sig
            hi = med + np.float32(n_sigma) * sig
            active = active & (row >= lo) & (row <= hi)
            med = np.float32(_lower_nanmedian(np.where(active, row, np.nan)))
            cnt = max(1, int(active.sum()))
            d = np.where(active, row - med, 0).astype(np.float32)
            sig = np.float32(np.sqrt(np.float32(np.sum(d * d, dtype=np.float64)) / np.float32(cnt)))
        out[r] = 0.0 if np.isnan(sig) else sig
    return out


# ---------------------------------------------------------------------------
# End-to-end streaming pipeline (services/corr_fast_integration.py:2063 corr +
# consume phases; services/cube_pipeline.py:2682 search cube), in the
# stream-time form the CUDA pipeline implements: time = absolute fast-vis tile.
# ---------------------------------------------------------------------------


def pipeline_tables(band: Band, antpos_e, antpos_n, *, nant, csf, n_grid, coarse_dm, fine_dm,
                    fine_to_coarse, t_int):
    G = band.n_chgroup
    cell = top_of_band_cell_lambda(antpos_e, antpos_n, band, n_grid)
    pats, cims = [], []
    for g in range(G):
        r, c = build_pattern(antpos_e, antpos_n, band, g, n_grid=n_grid, csf=csf, cell_lambda=cell)
        pats.append((r, c))
        cims.append(cell_index_map(antpos_e, antpos_n, band, g, n_grid=n_grid, csf=csf,
                                   cell_lambda=cell, ix_row_pat=r, ix_col_pat=c))
    t_int_us = t_int * NATIVE_SAMPLE_US
    sh1 = stage1_bin_shifts(band, coarse_dm, csf, t_int_us)                 # (G, C, K)
    sh2 = np.stack([stage2_shifts(band, g, coarse_dm, t_int_us) for g in range(G)])
    sf = time_shift_search(band, coarse_dm, fine_dm, fine_to_coarse, t_int_us, True)
    return dict(cell=cell, pats=pats, cims=cims, sh1=sh1, sh2=sh2, sf=sf)


def round_bf16(x: np.ndarray) -> np.ndarray:
    """float32 values rounded to the nearest bfloat16 (ties to even), returned
    as float32: the conversion of torch ``.to(torch.bfloat16)`` and of the
    stage-2 ring's BF16 storage form.  Keep the top 16 bits of the float32
    pattern after adding 0x7FFF plus the lowest kept bit; NaN stays NaN."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16).astype(np.uint32)
    out = r.view(np.float32).copy()
    nan = np.isnan(f)
    out[nan] = f[nan]
    return out


def round_bf16_complex(z: np.ndarray) -> np.ndarray:
    """complex64 with both parts rounded to bfloat16 (the BF16 ring element)."""
    z = np.asarray(z, np.complex64)
    return (round_bf16(z.real) + 1j * round_bf16(z.imag)).astype(np.complex64)


class Layer2State:
    """Per-kernel sigma_k of the detector's S/N (noise_norm/layer2.py:113-452)
    in its default configuration (no floor, no ratio clamp): seeded with
    sqrt(width) (detector/forward.py:746-755); a zero estimate keeps the
    previous value; Welford running mean over the first ``n_burnin`` cubes,
    then the EMA ``gamma * sigma + (1 - gamma) * s`` with gamma = 1 -
    exp(-cube_cadence_s / tau_s); float32 throughout."""

    def __init__(self, widths, cube_cadence_s: float, tau_s: float = 30.0, n_burnin: int = 30):
        self.s = np.asarray([math.sqrt(w) for w in widths], np.float32)
        self.gamma = 1.0 - math.exp(-cube_cadence_s / tau_s)
        self.n_burnin = int(n_burnin)
        self.count = 0

    def update(self, sigma: np.ndarray) -> np.ndarray:
        sig = np.asarray(sigma, np.float32)
        sig = np.where(sig == 0, self.s, sig).astype(np.float32)
        if self.count < self.n_burnin:
            c = np.float32(self.count)
            self.s = ((c * self.s + sig) / np.float32(self.count + 1.0)).astype(np.float32)
        else:
            self.s = (np.float32(self.gamma) * sig
                      + np.float32(1.0 - self.gamma) * self.s).astype(np.float32)
        self.count += 1
        return self.s


def layer2_sample_index(n_kernels: int, m: int, total: int) -> np.ndarray:
    """[K, m] flat indices over a cube interior of ``total`` cells: per kernel
    k, ``torch.randint(0, total, (m,))`` from a CPU generator seeded k
    (detector/forward.py:1436-1448)."""
    import torch
    out = np.empty((n_kernels, m), np.int64)
    for k in range(n_kernels):
        gen = torch.Generator(device="cpu")
        gen.manual_seed(int(k))
        out[k] = torch.randint(0, total, (m,), generator=gen).numpy()
    return out


def run_pipeline(raw_blocks, band: Band, antpos_e, antpos_n, *, nant, npkt_block, t_int, csf,
                 n_grid, coarse_dm, fine_dm, fine_to_coarse, log_max_width, threshold, chunk,
                 use_sky=True, sky_window=8, sky_warmup=8, n_top=None, r_t=4, r_f=5, r_lm=3,
                 l1_times=16, l1_pixels=256, ring_dtype="c64", keep=None, keep_images=True,
                 layer2=True, layer2_max_samples=4096, layer2_tau_s=30.0, layer2_n_burnin=30,
                 gains=None):
    """Oracle of the CUDA streaming pipeline; returns candidate tuples
    ``(t_abs, fdm, l, m, snr, width)`` and (optionally) intermediates.
    ``ring_dtype="bf16"`` stores the stage-2 streams in the BF16 form (each
    part rounded to bfloat16 after the sky subtraction), as the pipeline's
    precision form does; ``"cint8"`` sends every time row of every (chgroup,
    coarse DM) stream through the cint8 wire encoder (``encode_rows``, one
    tile per row) and stores what the receiver dequantises, float32(scale *
    q) per part."""
    keep = {} if keep is None else keep
    G = band.n_chgroup
    tb = pipeline_tables(band, antpos_e, antpos_n, nant=nant, csf=csf, n_grid=n_grid,
                         coarse_dm=coarse_dm, fine_dm=fine_dm, fine_to_coarse=fine_to_coarse,
                         t_int=t_int)
    n_coarse = len(coarse_dm)
    n_fine = len(fine_dm)
    N = n_grid
    # correlate every block -> integer vis stream per chgroup (T, nbase, C)
    vis = [[] for _ in range(G)]
    for blk in raw_blocks:
        for g in range(G):
            vr, vi = corr_fast_from_raw(blk[g].reshape(-1), npkt=npkt_block, nant=nant,
                                        nchan=band.nchan, t_int=t_int, csf=csf)
            vis[g].append(vr + 1j * vi)
    vis = [np.concatenate(v, axis=0) for v in vis]
    if gains is not None:
        # calibration as the voltages would carry it (apply_cal_split,
        # slow_corr_kernel.py:459) with one gain per antenna and summed
        # channel: V_ab -> g_a conj(g_b) V_ab, in float64
        ceff = band.nchan // csf
        gq = np.broadcast_to(np.asarray(gains, np.complex64), (G, ceff, nant)).astype(np.complex128)
        a_idx, b_idx = upper_tri_indices(nant)
        for g in range(G):
            vis[g] = vis[g] * (gq[g][:, a_idx] * np.conj(gq[g][:, b_idx])).T[None]
    T_total = vis[0].shape[0]
    max_sh1 = int(tb["sh1"].max())
    depth1 = -(-max_sh1 // chunk)
    n_chunks = T_total // chunk
    n_s1 = n_chunks - depth1                       # stage-1 chunks emitted
    sky = StaticSkyMean(sky_window, sky_warmup, n_dm=G * n_coarse) if use_sky else None
    # stage-1 output streams D1[g][d] (T1, n_filled)
    D1 = [[np.zeros((max(0, n_s1) * chunk, tb["pats"][g][0].size), np.complex128)
           for _ in range(n_coarse)] for g in range(G)]
    for j in range(max(0, n_s1)):
        for g in range(G):
            r, _ = tb["pats"][g]
            win = vis[g][j * chunk: (j + 1) * chunk + max_sh1]
            pad = (j + 1) * chunk + max_sh1 - j * chunk - win.shape[0]
            if pad > 0:
                win = np.concatenate([win, np.zeros((pad,) + win.shape[1:], win.dtype)])
            exact = (lambda x: np.rint(x).astype(np.int64)) if gains is None else (lambda x: x)
            o_re = stage1_dedisp(exact(win.real), tb["sh1"][g], tb["cims"][g], r.size, chunk)
            o_im = stage1_dedisp(exact(win.imag), tb["sh1"][g], tb["cims"][g], r.size, chunk)
            for d in range(n_coarse):
                x = (o_re[d] + 1j * o_im[d]).astype(np.complex64)
                if sky is not None:
                    x = sky.apply(x, dm_slot=g * n_coarse + d)
                if ring_dtype == "bf16":
                    x = round_bf16_complex(x)
                elif ring_dtype == "cint8":
                    x = decode_cint8(*encode_rows(x, 16))
                D1[g][d][j * chunk:(j + 1) * chunk] = x
    keep["D1"] = D1
    # search cubes
    L = max(0, -int(tb["sf"].min()))
    a = -(-L // chunk)
    te = (1 << log_max_width) // 2
    widths = [1 << k for k in range(log_max_width + 1)]
    if n_top is None:
        # the streaming decoder's rule (detector/forward.py:1383-1399, :1607)
        n_top = max(64, math.ceil(64 * (chunk + 2 * te) / chunk)) * len(widths)
    sinv = (np.float32(1.0) / np.sqrt(np.asarray(widths, np.float32))).astype(np.float32)
    offs = boxcar_offsets(widths, 1 << log_max_width)
    mask = edge_mask(N, kernel_support=1)
    act = np.nonzero(mask.reshape(-1) != 0)[0]
    l1_pix = act[np.linspace(0, act.size - 1, l1_pixels).astype(np.int64)]
    l1_t = te + np.linspace(0, chunk - 1, l1_times).astype(np.int64)
    T1 = max(0, n_s1) * chunk
    cands = []
    images = []
    l2 = None
    if layer2:
        # the streaming detector's Layer-2 path: S/N = boxcar / sigma_k of the
        # previous cube; the cube's score samples update sigma_k afterwards
        l2 = Layer2State(widths, chunk * t_int * NATIVE_SAMPLE_US * 1e-6, layer2_tau_s,
                         layer2_n_burnin)
        l2_idx = layer2_sample_index(len(widths), layer2_max_samples, chunk * n_fine * N * N)
        l2_t = l2_idx // (n_fine * N * N)
        l2_cell = l2_idx % (n_fine * N * N)
        l2_f, l2_p = l2_cell // (N * N), l2_cell % (N * N)
        l2_act = mask.reshape(-1)[l2_p] != 0
        keep["layer2_s"] = []
    # first cube whose every time has data from every chgroup (warm-up)
    jc_first = -(-(int(tb["sh2"].max()) + max(0, int(tb["sf"].max())) + 2 * te) // chunk)
    for jc in range(jc_first, max(0, n_s1 - a)):
        t0 = jc * chunk - 2 * te
        nt = chunk + 2 * te
        cube = np.zeros((nt, n_fine, N, N), np.float32)
        for f in range(n_fine):
            c = int(fine_to_coarse[f])
            img = np.zeros((nt, N, N), np.float64)
            # the combine of combine_half (sum over chgroups, Hermitian half,
            # checkerboard) a few times at a time, so that 512^2 cubes stay small
            for s0 in range(0, nt, 16):
                s1 = min(nt, s0 + 16)
                full = np.zeros((s1 - s0, N, N), np.complex128)
                for g in range(G):
                    r, cc = tb["pats"][g]
                    ri, ci = r.astype(np.int64), cc.astype(np.int64)
                    for t in range(s0, s1):
                        ts = t0 + t - int(tb["sf"][f, g]) - int(tb["sh2"][g, c])
                        if 0 <= ts < T1:
                            full[t - s0, ri, ci] += D1[g][c][ts]
                half = half_from_full(full, fftshift=True)
                img[s0:s1] = image_from_half(half, N)                   # float64
            img32 = img.astype(np.float32)
            samp = img32.reshape(nt, N * N)[l1_t][:, l1_pix].reshape(1, -1)
            sig = sigma_clipped_std_batched(samp)[0]
            sig = np.float32(sig if sig > 0 else 1.0)
            mf = (mask / sig).astype(np.float32)
            cube[:, f] = (img32 * mf[None]).astype(np.float32)
            if keep_images:
                images.append(img)
        score = np.zeros((chunk, n_fine, N, N), np.float32)
        win = np.zeros((chunk, n_fine, N, N), np.int16)
        if l2 is not None:
            sinv = (np.float32(1.0) / np.maximum(l2.s, np.float32(1e-30))).astype(np.float32)
            samp = np.full(l2_idx.shape, np.nan, np.float32)
        for r0 in range(0, N, 64):          # pixel-row slabs: the boxcars are per pixel
            cs = padded_cumsum(cube[:, :, r0:r0 + 64], 1 << log_max_width)
            score[:, :, r0:r0 + 64], win[:, :, r0:r0 + 64] = multi_boxcar_argmax(
                cs, widths, offs, sinv, chunk, te)
            if l2 is not None:
                # raw boxcar sums (before 1/sigma_k) at the sampled interior
                # cells of this slab, inside the edge mask
                csf = cs.reshape(cs.shape[0], n_fine, -1)
                for k, (w, off) in enumerate(zip(widths, offs)):
                    rows = l2_p[k] // N
                    sel = l2_act[k] & (rows >= r0) & (rows < r0 + 64)
                    pl = (rows[sel] - r0) * N + l2_p[k][sel] % N
                    tt = l2_t[k][sel] + te + off
                    samp[k, sel] = (csf[tt + w, l2_f[k][sel], pl]
                                    - csf[tt, l2_f[k][sel], pl]).astype(np.float32)
        if l2 is not None:
            keep["layer2_s"].append(l2.update(sigma_clipped_std_batched(samp)))
        for cd in decode_topk(score, win, threshold=threshold, n_top=n_top, r_t=r_t, r_f=r_f,
                              r_lm=r_lm):
            cands.append((jc * chunk - te + cd.t, cd.f, cd.l, cd.m, cd.snr, widths[cd.k]))
        if keep_images:
            keep.setdefault("cubes", []).append(cube)
    keep["images"] = images
    keep["tables"] = tb
    return cands
