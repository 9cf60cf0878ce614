"""Sparsity pattern and nearest-cell gridder — drop-in for
``dsart.grid.sparsity_pattern`` (build_pattern :893,
compute_top_of_band_cell_lambda :791) and ``dsart.grid.kernel.FastVisGridder``
(:108, from_pattern :234, compute :508).

The (u, v) -> cell arithmetic runs in FP64 on the GPU (``dsb_uv_cells``);
sorting/deduplicating the pattern keys and building the per-cell CSR source
lists are one-time host work, as in the reference.  K = 1 (nearest cell,
the reference's production default, constants.py KERNEL_SUPPORT_DEFAULT).
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib
from .constants import DSA110_BAND, SPEED_OF_LIGHT_M_S, Band, nbase_of

N_GRID_DEFAULT = 256


def _upper_tri(nants: int):
    a = np.repeat(np.arange(nants, dtype=np.int64), np.arange(1, nants + 1))
    b = np.concatenate([np.arange(k + 1, dtype=np.int64) for k in range(nants)])
    return a, b


def per_baseline_uv_meters(antpos_e, antpos_n, *, is_core_baseline_mask=None):
    """Kept cross baselines in bls order (sparsity_pattern.py:657-716).
    Returns ``(du_m, dv_m, keep_mask)``."""
    antpos_e = np.asarray(antpos_e, np.float64)
    antpos_n = np.asarray(antpos_n, np.float64)
    nants = antpos_e.shape[0]
    a, b = _upper_tri(nants)
    keep = a != b
    if is_core_baseline_mask is not None:
        m = np.asarray(is_core_baseline_mask, bool)
        if m.shape != (nbase_of(nants),):
            raise ValueError(f"is_core_baseline_mask shape {m.shape} != ({nbase_of(nants)},)")
        keep &= m
    return antpos_e[a[keep]] - antpos_e[b[keep]], antpos_n[a[keep]] - antpos_n[b[keep]], keep


def compute_top_of_band_cell_lambda(antpos_e, antpos_n, *, n_grid: int = N_GRID_DEFAULT,
                                    band: Band = DSA110_BAND,
                                    is_core_baseline_mask=None) -> float:
    """F28 common cell scale at the band top (sparsity_pattern.py:791-860)."""
    du, dv, _ = per_baseline_uv_meters(antpos_e, antpos_n,
                                       is_core_baseline_mask=is_core_baseline_mask)
    nu_top = float(band.freq_table()[0, 0])
    wl = SPEED_OF_LIGHT_M_S / (nu_top * 1e9)
    m = float(np.max(np.maximum(np.abs(du / wl), np.abs(dv / wl))))
    if m == 0.0:
        raise ValueError("max_baseline_lambda == 0 (degenerate antpos / mask)")
    return m * 2.0 / n_grid


def uv_cells_gpu(du: np.ndarray, dv: np.ndarray, nu_ghz: np.ndarray, cell_lambda: float,
                 n_grid: int, device) -> Tuple[np.ndarray, np.ndarray]:
    """FP64 cell coordinates on the GPU; returns host ``(row, col)`` int64
    arrays of shape ``(n_bl, n_ch)``."""
    dev = _lib.cuda_device(device)
    d_du = torch.from_numpy(np.ascontiguousarray(du, np.float64)).to(dev)
    d_dv = torch.from_numpy(np.ascontiguousarray(dv, np.float64)).to(dev)
    d_nu = torch.from_numpy(np.ascontiguousarray(nu_ghz, np.float64)).to(dev)
    n_bl, n_ch = du.shape[0], nu_ghz.shape[0]
    row = torch.empty((n_bl, n_ch), dtype=torch.int32, device=dev)
    col = torch.empty((n_bl, n_ch), dtype=torch.int32, device=dev)
    _lib.check(_lib.lib().dsb_uv_cells(_lib.ptr(d_du), _lib.ptr(d_dv), n_bl, _lib.ptr(d_nu), n_ch,
                                       float(cell_lambda), int(n_grid), _lib.ptr(row),
                                       _lib.ptr(col), _lib.stream_of(dev)), "dsb_uv_cells")
    return row.cpu().numpy().astype(np.int64), col.cpu().numpy().astype(np.int64)


@dataclass
class SparsityPattern:
    """Filled uv cells of one chgroup (sparsity_pattern.py:388): ``ix_row`` /
    ``ix_col`` uint16, sorted by the ``(row << 16) | col`` key."""

    ix_row: np.ndarray
    ix_col: np.ndarray
    n_grid: int
    chgroup: int
    chan_sum_factor: int
    cell_lambda: float
    kernel_support: int = 1
    band: Band = DSA110_BAND
    pattern_id: int = 0

    @property
    def n_filled(self) -> int:
        return int(self.ix_row.size)


def build_pattern(antpos_e, antpos_n, *, chgroup: int, dec_deg: float = 0.0,
                  n_grid: int = N_GRID_DEFAULT, kernel_support: int = 1,
                  chan_sum_factor: int = 1, cell_lambda: Optional[float] = None,
                  is_core_baseline_mask=None, band: Band = DSA110_BAND,
                  device="cuda") -> SparsityPattern:
    """Deterministic sparsity pattern for one chgroup (sparsity_pattern.py:893)."""
    if kernel_support != 1:
        raise ValueError("dsb200 grids with kernel_support=1 (nearest cell)")
    if not 0 <= chgroup < band.n_chgroup:
        raise ValueError(f"chgroup={chgroup} out of range 0..{band.n_chgroup - 1}")
    if chan_sum_factor < 1 or band.nchan % chan_sum_factor:
        raise ValueError(f"chan_sum_factor={chan_sum_factor} does not divide nchan={band.nchan}")
    if n_grid <= 0 or n_grid > 65535:
        raise ValueError(f"n_grid={n_grid} out of range")
    du, dv, _ = per_baseline_uv_meters(antpos_e, antpos_n,
                                       is_core_baseline_mask=is_core_baseline_mask)
    nu = band.summed_freq_table(chan_sum_factor)[chgroup]
    if cell_lambda is None:
        wl = SPEED_OF_LIGHT_M_S / (nu * 1e9)
        m = float(np.max(np.maximum(np.abs(du[:, None] / wl[None, :]),
                                    np.abs(dv[:, None] / wl[None, :]))))
        cell_lambda = m * 2.0 / n_grid
    row, col = uv_cells_gpu(du, dv, nu, cell_lambda, n_grid, device)
    ok = (row >= 0) & (row < n_grid) & (col >= 0) & (col < n_grid)
    keys = np.unique((row[ok].astype(np.uint32) << 16) | col[ok].astype(np.uint32))
    pid = int.from_bytes(hashlib.blake2b(keys.tobytes(), digest_size=8).digest(), "little")
    return SparsityPattern(ix_row=((keys >> 16) & 0xFFFF).astype(np.uint16),
                           ix_col=(keys & 0xFFFF).astype(np.uint16), n_grid=n_grid,
                           chgroup=chgroup, chan_sum_factor=chan_sum_factor,
                           cell_lambda=float(cell_lambda), band=band, pattern_id=pid)


def cell_index_map_for(pattern: SparsityPattern, antpos_e, antpos_n, *,
                       is_core_baseline_mask=None, device="cuda") -> np.ndarray:
    """``(nbase, nchan_eff)`` int64 filled-cell index, sentinel = n_filled
    (grid/kernel.py:308-470)."""
    nants = np.asarray(antpos_e).shape[0]
    du, dv, keep = per_baseline_uv_meters(antpos_e, antpos_n,
                                          is_core_baseline_mask=is_core_baseline_mask)
    nu = pattern.band.summed_freq_table(pattern.chan_sum_factor)[pattern.chgroup]
    row, col = uv_cells_gpu(du, dv, nu, pattern.cell_lambda, pattern.n_grid, device)
    n = pattern.n_grid
    ok = (row >= 0) & (row < n) & (col >= 0) & (col < n)
    pat_keys = (pattern.ix_row.astype(np.uint32) << 16) | pattern.ix_col.astype(np.uint32)
    keys = (np.where(ok, row, 0).astype(np.uint32) << 16) | np.where(ok, col, 0).astype(np.uint32)
    pos = np.searchsorted(pat_keys, keys)
    pos = np.where(ok, pos, pattern.n_filled)
    if np.any(ok & (pos >= pattern.n_filled)) or not np.all(
            pat_keys[np.minimum(pos[ok], pattern.n_filled - 1)] == keys[ok]):
        raise RuntimeError("in-grid cell missing from the pattern (geometry drift)")
    cim = np.full((nbase_of(nants), nu.shape[0]), pattern.n_filled, np.int64)
    cim[np.where(keep)[0]] = pos
    return cim


def cell_csr(cim: np.ndarray, n_filled: int) -> Tuple[np.ndarray, np.ndarray]:
    """Per-cell source lists (flat ``bls*C + s``, ascending) as int32 CSR."""
    flat = cim.reshape(-1)
    valid = np.nonzero(flat < n_filled)[0]
    order = valid[np.argsort(flat[valid], kind="stable")]
    counts = np.bincount(flat[valid], minlength=n_filled)
    off = np.zeros(n_filled + 1, np.int64)
    off[1:] = np.cumsum(counts)
    return off.astype(np.int32), order.astype(np.int32)


@dataclass
class FastVisGridder:
    """Nearest-cell gridder bound to one pattern (grid/kernel.py:108)."""

    pattern: SparsityPattern
    device: torch.device
    cell_index_map: torch.Tensor          # (nbase * nchan_eff,) int64 on the host
    cell_weights_cpu: torch.Tensor
    _off: torch.Tensor = field(init=False, repr=False)
    _src: torch.Tensor = field(init=False, repr=False)
    _w: torch.Tensor = field(init=False, repr=False)
    _nbase: int = field(init=False, repr=False)
    _nchan_eff: int = field(init=False, repr=False)

    def __post_init__(self) -> None:
        self.device = _lib.cuda_device(self.device)
        cim = self.cell_index_map.numpy()
        self._nchan_eff = self.pattern.band.nchan // self.pattern.chan_sum_factor
        self._nbase = cim.size // self._nchan_eff
        off, src = cell_csr(cim.reshape(self._nbase, self._nchan_eff), self.pattern.n_filled)
        self._off = torch.from_numpy(off).to(self.device)
        self._src = torch.from_numpy(src).to(self.device)
        self._w = self.cell_weights_cpu.to(self.device)

    @classmethod
    def from_pattern(cls, pattern: SparsityPattern, antpos_e, antpos_n, *,
                     is_core_baseline_mask=None, device="cuda") -> "FastVisGridder":
        cim = cell_index_map_for(pattern, antpos_e, antpos_n,
                                 is_core_baseline_mask=is_core_baseline_mask, device=device)
        flat = cim.reshape(-1)
        w = np.bincount(flat[flat < pattern.n_filled], minlength=pattern.n_filled)
        return cls(pattern=pattern, device=device, cell_index_map=torch.from_numpy(flat),
                   cell_weights_cpu=torch.from_numpy(w.astype(np.float32)))

    @property
    def cell_weights(self) -> torch.Tensor:
        """(n_filled,) float32 sum of squared tap weights (= hit count for K=1)."""
        return self._w

    @property
    def csr(self) -> Tuple[torch.Tensor, torch.Tensor]:
        return self._off, self._src

    def compute(self, vis_stokes_i: torch.Tensor) -> torch.Tensor:
        if not vis_stokes_i.is_complex():
            raise TypeError(f"vis_stokes_i must be complex; got {vis_stokes_i.dtype}")
        if vis_stokes_i.ndim != 3:
            raise ValueError(f"vis_stokes_i must be 3D (n_fast_vis, NBASE, NCHAN); got "
                             f"{vis_stokes_i.ndim}D shape {tuple(vis_stokes_i.shape)}")
        n_fv, nb, nch = vis_stokes_i.shape
        if nb != self._nbase:
            raise ValueError(f"vis_stokes_i.shape[1]={nb} != NBASE={self._nbase}")
        if nch != self._nchan_eff:
            raise ValueError(f"vis_stokes_i.shape[2]={nch} != NCHAN_eff={self._nchan_eff}")
        if vis_stokes_i.device != self.device:
            raise ValueError(f"vis_stokes_i on {vis_stokes_i.device}, gridder on {self.device}")
        v = vis_stokes_i.to(torch.complex64).contiguous()
        out = torch.empty((n_fv, self.pattern.n_filled), dtype=torch.complex64, device=self.device)
        _lib.check(_lib.lib().dsb_grid_vis(_lib.ptr(v), n_fv, nb * nch, _lib.ptr(self._off),
                                           _lib.ptr(self._src), self.pattern.n_filled,
                                           _lib.ptr(out), _lib.stream_of(self.device)),
                   "dsb_grid_vis")
        return out
