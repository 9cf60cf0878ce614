"""Candidate post-processing after the detector.

This module holds the cross-kernel merger (detector/merger.py:78-276) and
the canonical-zone emit gate (detector/decoder.py:541-636) of the reference.
They work on lists of the reference's ``Candidate`` records, or on any
dataclass with the same fields: ``l, m, dm_fine, dm_idx, event_specnum,
width_samples, kernel_id, snr, flags``.  Survivors and emitted candidates
are returned as the same objects; dropped ones are copies with their flag
bits set.

Both mergers sort by (SNR descending, event_specnum, dm_idx, l, m,
kernel_id).  They keep a candidate unless an earlier survivor lies inside
its neighbourhood:
* C1 rule: |dt| within half the summed widths (x t_frac x the spec-num
  period), |d dm_idx| <= dm_max_trials, and |dl| OR |dm| <= lm_max_cells
  (the DSA core's cross-shaped PSF);
* legacy rule: a box on all four axes.

The survivors' coordinates are kept in arrays, so each candidate is tested
against all of them at once.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

NOISE_WARMUP = 1 << 3
RFI_WARMING_UP = 1 << 4
HALO_DROPPED = 1 << 5       # dm_idx outside this node's canonical range
TIME_EDGE_DROPPED = 1 << 6  # inside the first or last n_kernel_max_t // 2 samples

DEFAULT_MERGE_RADIUS_LM = 3
DEFAULT_MERGE_RADIUS_FDM = 5
DEFAULT_MERGE_RADIUS_T = 128


@dataclass(frozen=True)
class MergerConfig:
    """C1 merger geometry (the reference's MergerConfig defaults)."""

    lm_max_cells: int = 3
    dm_max_trials: int = 2
    t_frac: float = 1.0
    sample_period_specnum: int = 16

    def __post_init__(self) -> None:
        if self.lm_max_cells < 0:
            raise ValueError(f"lm_max_cells={self.lm_max_cells}, expected ≥ 0")
        if self.dm_max_trials < 0:
            raise ValueError(f"dm_max_trials={self.dm_max_trials}, expected ≥ 0")
        if self.t_frac < 0.0:
            raise ValueError(f"t_frac={self.t_frac}, expected ≥ 0")
        if self.sample_period_specnum <= 0:
            raise ValueError(
                f"sample_period_specnum={self.sample_period_specnum}, expected > 0")


def _sorted(candidates: Sequence) -> list:
    return sorted(candidates, key=lambda c: (-c.snr, c.event_specnum, c.dm_idx, c.l, c.m,
                                             c.kernel_id))


class _Survivors:
    """Coordinates of the survivors so far, grown in place."""

    def __init__(self, n: int):
        self.t = np.empty(n, np.int64)
        self.d = np.empty(n, np.int64)
        self.w = np.empty(n, np.int64)
        self.l = np.empty(n, np.float64)
        self.m = np.empty(n, np.float64)
        self.n = 0

    def add(self, c) -> None:
        k = self.n
        self.t[k], self.d[k], self.w[k] = int(c.event_specnum), int(c.dm_idx), int(c.width_samples)
        self.l[k], self.m[k] = float(c.l), float(c.m)
        self.n = k + 1


def merge_across_kernels_c1(candidates: Sequence, cfg: MergerConfig) -> List:
    """C1 cross-kernel merger (merger.py:123-197): see the module notes."""
    if not candidates:
        return []
    order = _sorted(candidates)
    lm, dmx = float(int(cfg.lm_max_cells)), int(cfg.dm_max_trials)
    half = float(cfg.t_frac) * 0.5
    sps = float(cfg.sample_period_specnum)
    sv = _Survivors(len(order))
    out = []
    for c in order:
        k = sv.n
        if k:
            # dt <= t_frac * 0.5 * (w_c + w_s) * sps, evaluated in that order
            dt_max = half * (int(c.width_samples) + sv.w[:k]).astype(np.float64) * sps
            hit = ((np.abs(int(c.event_specnum) - sv.t[:k]) <= dt_max)
                   & (np.abs(int(c.dm_idx) - sv.d[:k]) <= dmx)
                   & ((np.abs(float(c.l) - sv.l[:k]) <= lm) | (np.abs(float(c.m) - sv.m[:k]) <= lm)))
            if hit.any():
                continue
        sv.add(c)
        out.append(c)
    return out


def merge_across_kernels(candidates: Sequence, *, merge_radius_lm: int = DEFAULT_MERGE_RADIUS_LM,
                         merge_radius_fdm: int = DEFAULT_MERGE_RADIUS_FDM,
                         merge_radius_t: int = DEFAULT_MERGE_RADIUS_T) -> List:
    """Legacy merger (merger.py:217-276): suppressed only when within every
    radius on (t, dm_idx, l, m)."""
    if merge_radius_lm < 0 or merge_radius_fdm < 0 or merge_radius_t < 0:
        raise ValueError(f"merge_radius_lm/fdm/t must be ≥ 0; got "
                         f"({merge_radius_lm}, {merge_radius_fdm}, {merge_radius_t})")
    if not candidates:
        return []
    order = _sorted(candidates)
    sv = _Survivors(len(order))
    out = []
    for c in order:
        k = sv.n
        if k:
            hit = ((np.abs(int(c.event_specnum) - sv.t[:k]) <= merge_radius_t)
                   & (np.abs(int(c.dm_idx) - sv.d[:k]) <= merge_radius_fdm)
                   & (np.abs(c.l - sv.l[:k]) <= merge_radius_lm)
                   & (np.abs(c.m - sv.m[:k]) <= merge_radius_lm))
            if hit.any():
                continue
        sv.add(c)
        out.append(c)
    return out


def filter_to_canonical(candidates: Sequence, *, dm_idx_canonical_lo: int,
                        dm_idx_canonical_hi: int, t_det: int, n_kernel_max_t: int,
                        cube_t_offset: int = 0) -> Tuple[List, List]:
    """Canonical-zone emit gate (decoder.py:541-636): ``(emit, dropped)``.
    A candidate outside ``[dm_idx_canonical_lo, dm_idx_canonical_hi]`` gets
    HALO_DROPPED.  One whose cube time ``event_specnum - cube_t_offset`` is
    outside ``[n_kernel_max_t // 2, t_det - n_kernel_max_t // 2)`` gets
    TIME_EDGE_DROPPED.  Dropped candidates are copies with those bits added;
    other flag bits pass through."""
    if dm_idx_canonical_hi < dm_idx_canonical_lo:
        raise ValueError(f"dm_idx_canonical_hi={dm_idx_canonical_hi} < "
                         f"dm_idx_canonical_lo={dm_idx_canonical_lo}")
    if t_det < 1 or n_kernel_max_t < 1:
        raise ValueError(f"t_det={t_det} / n_kernel_max_t={n_kernel_max_t} must both be ≥ 1")
    lo_t, hi_t = n_kernel_max_t // 2, t_det - n_kernel_max_t // 2
    emit, dropped = [], []
    for c in candidates:
        bits = 0
        if not dm_idx_canonical_lo <= c.dm_idx <= dm_idx_canonical_hi:
            bits |= HALO_DROPPED
        if not lo_t <= int(c.event_specnum) - int(cube_t_offset) < hi_t:
            bits |= TIME_EDGE_DROPPED
        flags = int(c.flags) | bits
        if flags == int(c.flags):
            emit.append(c)
        else:
            dropped.append(dataclasses.replace(c, flags=flags))
    return emit, dropped
