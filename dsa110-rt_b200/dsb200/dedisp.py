"""Coarse/fine dedispersion plan, stage 1, static sky and stage-2 FIFOs —
drop-in for ``dsart.coarse_dm`` (dm_plan.py, stage1.py,
stage2_shifts.py, stage2_fifo.py, stage2_per_dm_fifo.py,
stage2_chgroup_alignment.py), ``Stage1MultiDMCoarseDM`` / ``StaticSkyMean``
(services/corr_fast_integration.py:495, :1049) and
``dsart.fine_dm.combiner.compute_time_shift_search`` (:150).

Shift tables are FP64 host arithmetic with ``np.rint`` (half to even), the
same operation order as the reference; everything per-sample runs in
``libdsb200.so`` on the device.
"""

from __future__ import annotations

from collections import deque
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .constants import DSA110_BAND, K_DM_MS_GHZ2_PC, NATIVE_SAMPLE_US, Band


def delta_tau_us(nu_low: float, nu_high: float, dm: float) -> float:
    """common/dispersion.py:39-66."""
    ms = K_DM_MS_GHZ2_PC * dm * (1.0 / (nu_low * nu_low) - 1.0 / (nu_high * nu_high))
    return 1000.0 * ms


def compute_delay_native_samples_table(coarse_dm: np.ndarray, chgroup_freqs_GHz: np.ndarray
                                       ) -> np.ndarray:
    """``(G, C, K)`` int64 delays in native samples, Convention A
    (coarse_dm/dm_plan.py:194-243)."""
    nu = np.asarray(chgroup_freqs_GHz, np.float64)
    nu_top = nu[:, 0:1]
    inv_diff = (1.0 / (nu ** 2)) - (1.0 / (nu_top ** 2))
    delay_us = (K_DM_MS_GHZ2_PC * np.asarray(coarse_dm, np.float64)[None, None, :]
                * inv_diff[:, :, None] * 1e3)
    return np.rint(delay_us / NATIVE_SAMPLE_US).astype(np.int64)


@dataclass(frozen=True)
class DMPlan:
    """Coarse-DM plan over summed channels (dm_plan.py:244-700)."""

    dm_pc_cc: np.ndarray
    t_int_fast_us: float
    chan_sum_factor: int = 1
    band: Band = DSA110_BAND
    n_fine_per_coarse: int = 1

    @property
    def n_coarse(self) -> int:
        return int(self.dm_pc_cc.shape[0])

    @property
    def chgroup_freqs_GHz(self) -> np.ndarray:
        return self.band.summed_freq_table(self.chan_sum_factor)

    @property
    def t_int_fast_native(self) -> float:
        return float(self.t_int_fast_us) / NATIVE_SAMPLE_US

    def delay_native_samples_per_chgroup(self, chgroup: int) -> np.ndarray:
        return compute_delay_native_samples_table(self.dm_pc_cc, self.chgroup_freqs_GHz)[chgroup]

    def delay_bins_per_chgroup(self, chgroup: int) -> np.ndarray:
        nat = self.delay_native_samples_per_chgroup(chgroup)
        return np.rint(nat / self.t_int_fast_native).astype(np.int64)

    def delay_bins_all(self) -> np.ndarray:
        """``(G, C_eff, K)`` int64."""
        nat = compute_delay_native_samples_table(self.dm_pc_cc, self.chgroup_freqs_GHz)
        return np.rint(nat / self.t_int_fast_native).astype(np.int64)


def max_t_dedisp_for_plan(n_fast_vis: int, plan: DMPlan, *, chgroup: int,
                          dm_indices: Optional[np.ndarray] = None) -> int:
    """coarse_dm/stage1.py:111."""
    b = plan.delay_bins_per_chgroup(chgroup)
    if dm_indices is not None:
        b = b[:, np.asarray(dm_indices, np.int64)]
    return max(0, int(n_fast_vis) - (int(b.max()) if b.size else 0))


@dataclass(frozen=True)
class Stage2ShiftTable:
    chgroup: int
    coarse_dm_pc_cm3: np.ndarray
    nu_chgroup_ref_GHz: float
    nu_bot_proc_GHz: float
    t_int_corr_us: float
    shifts_samples: np.ndarray

    @property
    def n_coarse(self) -> int:
        return int(self.shifts_samples.shape[0])

    @property
    def max_shift(self) -> int:
        return int(self.shifts_samples.max())


def compute_stage2_shifts(*, chgroup: int, coarse_dm_pc_cm3: np.ndarray,
                          t_int_corr_us: float = 262.144, band: Band = DSA110_BAND
                          ) -> Stage2ShiftTable:
    """``rint(dtau(nu_bot_proc, nu_top[g], dm_c) / t_int)`` (stage2_shifts.py:170-321)."""
    if not 0 <= chgroup < band.n_chgroup:
        raise ValueError(f"chgroup={chgroup} out of range [0, {band.n_chgroup})")
    cd = np.asarray(coarse_dm_pc_cm3, np.float64)
    if cd.ndim != 1:
        raise ValueError(f"coarse_dm_pc_cm3 must be 1D, got ndim={cd.ndim}")
    if np.any(cd < 0):
        raise ValueError("coarse_dm_pc_cm3 contains negative entries")
    if t_int_corr_us <= 0:
        raise ValueError(f"t_int_corr_us={t_int_corr_us} must be > 0")
    nu_bot = band.bot_proc()
    nu_g = float(band.chgroup_top()[chgroup])
    sh = np.asarray([int(np.rint(delta_tau_us(nu_bot, nu_g, float(d)) / t_int_corr_us))
                     for d in cd], np.int32)
    return Stage2ShiftTable(chgroup, cd, nu_g, nu_bot, float(t_int_corr_us), sh)


def compute_time_shift_search(*, coarse_dm_pc_cm3, fine_dm_pc_cm3, fine_to_coarse,
                              t_int_search_us: float, merge_coarse_rounding: bool = True,
                              band: Band = DSA110_BAND) -> np.ndarray:
    """Signed int32 ``(N_fine, G)`` residual shifts, chgroup-TOP reference
    (fine_dm/combiner.py:150-498; merged rounding is the production flag)."""
    tops = band.chgroup_top()
    nu_bot = band.bot_proc()
    cd = np.asarray(coarse_dm_pc_cm3, np.float64)
    fd = np.asarray(fine_dm_pc_cm3, np.float64)
    f2c = np.asarray(fine_to_coarse, np.int64)
    if f2c.shape != fd.shape:
        raise ValueError("fine_to_coarse and fine_dm lengths differ")
    out = np.zeros((fd.size, tops.size), np.int32)
    for f in range(fd.size):
        c = int(f2c[f])
        for g in range(tops.size):
            if merge_coarse_rounding:
                s_f = np.rint(delta_tau_us(nu_bot, float(tops[g]), float(fd[f])) / t_int_search_us)
                s_c = np.rint(delta_tau_us(nu_bot, float(tops[g]), float(cd[c])) / t_int_search_us)
                out[f, g] = int(s_f - s_c)
            else:
                out[f, g] = int(np.rint(delta_tau_us(nu_bot, float(tops[g]),
                                                     float(fd[f] - cd[c])) / t_int_search_us))
    return out


# ---------------------------------------------------------------------------
# Stage 1 (vis-domain shift + grid), reference call surface
# ---------------------------------------------------------------------------


@dataclass
class Stage1MultiDMCoarseDM:
    """Per-DM stage-1 shift + grid (corr_fast_integration.py:495-1046).

    ``sliding_window=True`` is F34: the first call emits zeros, later calls
    emit the previous block dedispersed against previous + current."""

    plan: DMPlan
    gridder: "object"
    chgroup: int
    dm_indices: Optional[np.ndarray] = None
    sliding_window: bool = False
    dm_chunk_size: int = 2
    _prev: Optional[torch.Tensor] = field(default=None, init=False, repr=False)
    _shifts_dev: Optional[torch.Tensor] = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        if not 0 <= self.chgroup < self.plan.band.n_chgroup:
            raise ValueError(f"Stage1MultiDMCoarseDM.chgroup={self.chgroup}, expected "
                             f"0..{self.plan.band.n_chgroup - 1}")
        if self.dm_indices is None:
            self._idx = np.arange(self.plan.n_coarse, dtype=np.int64)
        else:
            arr = np.asarray(self.dm_indices, np.int64).reshape(-1)
            if arr.size == 0:
                raise ValueError("dm_indices is empty")
            if int(arr.min()) < 0 or int(arr.max()) >= self.plan.n_coarse:
                raise IndexError(f"dm_indices contain out-of-range trials "
                                 f"(plan.n_coarse={self.plan.n_coarse})")
            self._idx = arr
        self._bins = self.plan.delay_bins_per_chgroup(self.chgroup)[:, self._idx]

    @property
    def n_dm(self) -> int:
        return int(self._idx.shape[0])

    @property
    def n_filled_out(self) -> int:
        return int(self.gridder.pattern.n_filled)

    def t_dedisp_for(self, n_fast_vis: int) -> int:
        return max(0, int(n_fast_vis) - int(self._bins.max()))

    def _shifts(self, dev) -> torch.Tensor:
        if self._shifts_dev is None:
            self._shifts_dev = torch.from_numpy(
                np.ascontiguousarray(self._bins.astype(np.int32))).to(dev)
        return self._shifts_dev

    def _window(self, prev: Optional[torch.Tensor], cur: torch.Tensor, t_out: int) -> torch.Tensor:
        dev = cur.device
        n_prev = 0 if prev is None else int(prev.shape[0])
        _, nb, nch = cur.shape
        off, src = self.gridder.csr
        out = torch.empty((self.n_dm, t_out, self.n_filled_out), dtype=torch.complex64,
                          device=dev)
        _lib.check(_lib.lib().dsb_dedisp_vis(
            _lib.ptr(prev), _lib.ptr(cur), n_prev, nb * nch, nch, _lib.ptr(off), _lib.ptr(src),
            _lib.ptr(self._shifts(dev)), self.n_dm, self.n_filled_out, t_out, _lib.ptr(out),
            _lib.stream_of(dev)), "dsb_dedisp_vis")
        return out

    def dedisperse_from_vis(self, vis_stokes_i: torch.Tensor, *, block_n: int) -> torch.Tensor:
        if vis_stokes_i.ndim != 3:
            raise ValueError(f"vis_stokes_i must be 3-D (n_fv, NBASE, NCHAN); got "
                             f"{vis_stokes_i.ndim}-D shape {tuple(vis_stokes_i.shape)}")
        _lib.require_cuda(vis_stokes_i, "vis_stokes_i")
        v = vis_stokes_i.to(torch.complex64)
        n_fv = int(v.shape[0])
        if not self.sliding_window:
            t_d = self.t_dedisp_for(n_fv)
            if t_d <= 0:
                raise ValueError(f"n_fast_vis={n_fv} too short for plan max bin shift on "
                                 f"chgroup={self.chgroup}")
            return self._window(None, v, t_d)
        if self._prev is None:
            self._prev = v.clone()
            return torch.zeros((self.n_dm, n_fv, self.n_filled_out), dtype=torch.complex64,
                               device=v.device)
        if int(self._prev.shape[0]) != n_fv:
            raise ValueError(f"sliding-window: prev block n_fv={int(self._prev.shape[0])} != "
                             f"current n_fv={n_fv}; F34 assumes uniform-block streams")
        if 2 * n_fv - int(self._bins.max()) < n_fv:
            raise ValueError(f"sliding-window: max plan shift ({int(self._bins.max())}) exceeds "
                             f"prev-block n_fv={n_fv}; bump ring-buffer K above 2.")
        out = self._window(self._prev, v, n_fv)
        self._prev = v.clone()
        return out


# ---------------------------------------------------------------------------
# Static sky (reference call surface)
# ---------------------------------------------------------------------------


@dataclass
class StaticSkyMean:
    """Boxcar mean of the past ``window_blocks`` cubes' per-cell means
    (corr_fast_integration.py:1049-1240); state lives on the device in float64."""

    window_blocks: int = 8
    warmup_cubes: int = 8
    n_dm: int = 1

    def __post_init__(self) -> None:
        if self.window_blocks < 1:
            raise ValueError(f"StaticSkyMean.window_blocks={self.window_blocks}, expected >= 1")
        if self.warmup_cubes < 0:
            raise ValueError(f"StaticSkyMean.warmup_cubes={self.warmup_cubes}, expected >= 0")
        if self.n_dm < 1:
            raise ValueError(f"StaticSkyMean.n_dm={self.n_dm}, expected >= 1")
        self.reset()

    def reset(self) -> None:
        self._ring: List[Optional[torch.Tensor]] = [None] * self.n_dm
        self._count = [0] * self.n_dm
        self._head = [0] * self.n_dm
        self._seen = [0] * self.n_dm

    def cubes_seen_for(self, dm_slot: int = 0) -> int:
        return int(self._seen[dm_slot])

    def in_warmup_for(self, dm_slot: int = 0) -> bool:
        return self._seen[dm_slot] < self.warmup_cubes

    def apply(self, gridded: torch.Tensor, dm_slot: int = 0) -> torch.Tensor:
        if not gridded.is_complex():
            raise TypeError(f"StaticSkyMean.apply: gridded must be complex; got {gridded.dtype}")
        if gridded.ndim != 2:
            raise ValueError(f"StaticSkyMean.apply: gridded must be 2D (n_fast_vis, N_filled); "
                             f"got {tuple(gridded.shape)}")
        s = int(dm_slot)
        if s < 0 or s >= self.n_dm:
            raise IndexError(f"StaticSkyMean.apply: dm_slot={s} out of range [0, {self.n_dm})")
        _lib.require_cuda(gridded, "gridded")
        g = gridded.to(torch.complex64).contiguous()
        n_t, n_cells = g.shape
        if self._ring[s] is None:
            self._ring[s] = torch.zeros((n_cells, self.window_blocks), dtype=torch.complex128,
                                        device=g.device)
        out = torch.empty_like(g)
        subtract = int(self._count[s] > 0 and self._seen[s] >= self.warmup_cubes)
        _lib.check(_lib.lib().dsb_static_sky(_lib.ptr(g), _lib.ptr(out), n_t, n_cells,
                                             _lib.ptr(self._ring[s]), self.window_blocks,
                                             self._head[s], self._count[s], subtract,
                                             _lib.stream_of(g.device)), "dsb_static_sky")
        if self._count[s] < self.window_blocks:
            self._count[s] += 1
        self._head[s] = (self._head[s] + 1) % self.window_blocks
        self._seen[s] += 1
        return out


# ---------------------------------------------------------------------------
# Stage-2 FIFOs (reference call surface)
# ---------------------------------------------------------------------------


class Stage2FIFO:
    """Bounded oldest-evicting FIFO of cube references (stage2_fifo.py:83-305)."""

    def __init__(self, depth: int = 4) -> None:
        if depth < 1:
            raise ValueError(f"depth={depth}, expected ≥ 1")
        self._depth = int(depth)
        self._buf: deque = deque()
        self._ref = None

    @property
    def depth(self) -> int:
        return self._depth

    def __len__(self) -> int:
        return len(self._buf)

    def empty(self) -> bool:
        return not self._buf

    def full(self) -> bool:
        return len(self._buf) == self._depth

    def _pin(self, cube: torch.Tensor, who: str) -> None:
        if not isinstance(cube, torch.Tensor):
            raise TypeError(f"{who} expected torch.Tensor; got {type(cube).__name__}")
        if self._ref is None:
            self._ref = (tuple(cube.shape), cube.dtype, cube.device)
            return
        shape, dtype, device = self._ref
        if tuple(cube.shape) != shape:
            raise ValueError(f"{who} cube shape={tuple(cube.shape)} != first-push shape={shape}")
        if cube.dtype != dtype:
            raise ValueError(f"{who} cube dtype={cube.dtype} != first-push dtype={dtype}")
        if cube.device != device:
            raise ValueError(f"{who} cube device={cube.device} != first-push device={device}")

    def push(self, cube: torch.Tensor) -> Optional[torch.Tensor]:
        self._pin(cube, "Stage2FIFO.push")
        ev = self._buf.popleft() if len(self._buf) == self._depth else None
        self._buf.append(cube)
        return ev

    def push_for_protocol(self, cube: torch.Tensor, *, block_n: int = 0) -> list:
        ev = self.push(cube)
        return [] if ev is None else [ev]

    def peek_latest(self):
        return self._buf[-1] if self._buf else None

    def peek_oldest(self):
        return self._buf[0] if self._buf else None

    def as_list(self) -> list:
        return list(self._buf)

    def __iter__(self):
        return iter(self._buf)

    def clear(self) -> None:
        self._buf.clear()
        self._ref = None


class PerCoarseDmStage2FIFO:
    """Depth D per coarse DM: push i emits push i-D (stage2_per_dm_fifo.py:108-286)."""

    def __init__(self, depths_per_coarse_dm: Sequence[int]) -> None:
        d = [int(x) for x in depths_per_coarse_dm]
        if not d:
            raise ValueError("depths_per_coarse_dm is empty")
        if any(x < 0 for x in d):
            raise ValueError("depths must be >= 0")
        self._depths = d
        self._bufs = [deque() if x > 0 else None for x in d]
        self._ref: List = [None] * len(d)

    @property
    def n_coarse(self) -> int:
        return len(self._depths)

    @property
    def depths(self) -> tuple:
        return tuple(self._depths)

    def __len__(self) -> int:
        return sum(0 if b is None else len(b) for b in self._bufs)

    def occupancy(self, c: int) -> int:
        b = self._bufs[c]
        return 0 if b is None else len(b)

    def push(self, coarse_dm_index: int, slice_: torch.Tensor) -> Optional[torch.Tensor]:
        if not isinstance(slice_, torch.Tensor):
            raise TypeError(f"PerCoarseDmStage2FIFO.push expected torch.Tensor; got "
                            f"{type(slice_).__name__}")
        c = int(coarse_dm_index)
        if c < 0 or c >= self.n_coarse:
            raise ValueError(f"coarse_dm_index={c} out of range [0, {self.n_coarse})")
        key = (tuple(slice_.shape), slice_.dtype, slice_.device)
        if self._ref[c] is None:
            self._ref[c] = key
        elif key != self._ref[c]:
            raise ValueError(f"coarse_dm={c}: slice (shape, dtype, device) {key} != first-push "
                             f"{self._ref[c]}")
        d, buf = self._depths[c], self._bufs[c]
        if d == 0 or buf is None:
            return slice_
        if len(buf) < d:
            buf.append(slice_)
            return None
        out = buf.popleft()
        buf.append(slice_)
        return out

    def flush(self, c: int) -> list:
        buf = self._bufs[c]
        if buf is None:
            return []
        out = list(buf)
        buf.clear()
        return out

    def __iter__(self):
        for c in range(self.n_coarse):
            yield c, self.occupancy(c), self._depths[c]


class Stage2InterChgroupShiftFifo:
    """Per-coarse-DM time roll with whole-cube warm-up gating
    (stage2_chgroup_alignment.py:79-338).  History is held on the device and
    the aligned cube is assembled by one kernel launch."""

    def __init__(self, *, chgroup: int, coarse_dm_pc_cm3: np.ndarray, t_dedisp: int,
                 t_int_corr_us: float = 262.144, shift_table: Optional[Stage2ShiftTable] = None,
                 band: Band = DSA110_BAND) -> None:
        if t_dedisp < 1:
            raise ValueError(f"t_dedisp={t_dedisp} must be >= 1")
        if shift_table is None:
            shift_table = compute_stage2_shifts(chgroup=chgroup,
                                                coarse_dm_pc_cm3=coarse_dm_pc_cm3,
                                                t_int_corr_us=t_int_corr_us, band=band)
        elif shift_table.chgroup != chgroup:
            raise ValueError(f"shift_table.chgroup={shift_table.chgroup} != chgroup arg={chgroup}")
        self._chgroup = int(chgroup)
        self._T = int(t_dedisp)
        sh = shift_table.shifts_samples.astype(np.int64)
        self._shifts = sh
        self._k = sh // self._T
        self._r = sh - self._k * self._T
        self._n_dm = int(sh.size)
        self._depth = int(self._k.max()) + 2
        self._hist: deque = deque(maxlen=self._depth)
        self._pushed = 0
        self._ref = None
        self._dev_tabs = None

    @property
    def chgroup(self) -> int:
        return self._chgroup

    @property
    def t_dedisp(self) -> int:
        return self._T

    @property
    def n_dm(self) -> int:
        return self._n_dm

    @property
    def shifts_samples(self) -> np.ndarray:
        return self._shifts

    def _required(self) -> np.ndarray:
        return self._k + 1 + (self._r > 0)

    def per_dm_warmed(self) -> list:
        return [bool(min(self._pushed, self._depth) >= r) for r in self._required()]

    def warmed_up(self) -> bool:
        return all(self.per_dm_warmed())

    def any_warmed_up(self) -> bool:
        return any(self.per_dm_warmed())

    def push(self, dedispersed: torch.Tensor, *, block_n: int) -> list:
        if not isinstance(dedispersed, torch.Tensor):
            raise TypeError("Stage2InterChgroupShiftFifo.push expected torch.Tensor; "
                            f"got {type(dedispersed).__name__}")
        if dedispersed.ndim != 3:
            raise ValueError(f"dedispersed.ndim={dedispersed.ndim}, expected 3 "
                             f"(N_DM, T_dedisp, N_filled)")
        n_dm_in, t_in, _ = dedispersed.shape
        if n_dm_in != self._n_dm:
            raise ValueError(f"dedispersed.shape[0]={n_dm_in} != n_dm={self._n_dm}")
        if t_in != self._T:
            raise ValueError(f"dedispersed.shape[1]={t_in} != t_dedisp={self._T}")
        if self._ref is None:
            self._ref = (dedispersed.dtype, dedispersed.device)
        else:
            if dedispersed.dtype != self._ref[0]:
                raise ValueError(f"dedispersed.dtype={dedispersed.dtype} != first-push dtype="
                                 f"{self._ref[0]}")
            if dedispersed.device != self._ref[1]:
                raise ValueError(f"dedispersed.device={dedispersed.device} != first-push device="
                                 f"{self._ref[1]}")
        _lib.require_cuda(dedispersed, "dedispersed")
        if dedispersed.dtype != torch.complex64:
            raise ValueError("dsb200 stage-2 FIFO carries complex64 cubes")
        self._hist.appendleft(dedispersed.contiguous())
        self._pushed += 1
        warm = self.per_dm_warmed()
        if not any(warm):
            return []
        dev = dedispersed.device
        if self._dev_tabs is None:
            self._dev_tabs = (torch.from_numpy(self._k.astype(np.int32)).to(dev),
                              torch.from_numpy(self._r.astype(np.int32)).to(dev))
        ptrs = torch.tensor([h.data_ptr() for h in self._hist], dtype=torch.int64).to(dev)
        w = torch.tensor([int(x) for x in warm], dtype=torch.int32).to(dev)
        out = torch.empty_like(dedispersed)
        inner = int(dedispersed.shape[2])
        _lib.check(_lib.lib().dsb_stage2_roll(_lib.ptr(ptrs), len(self._hist),
                                              _lib.ptr(self._dev_tabs[0]),
                                              _lib.ptr(self._dev_tabs[1]), _lib.ptr(w),
                                              self._n_dm, self._T, inner, _lib.ptr(out),
                                              _lib.stream_of(dev)), "dsb_stage2_roll")
        return [out]
