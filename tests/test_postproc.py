"""Candidate post-processing (detector/merger.py:78-276,
detector/decoder.py:541-636): the C1 and legacy cross-kernel mergers and
the canonical-zone gate equal the reference's output on seeded clustered
candidates (tests/golden/make_golden.py), survivor for survivor and flag
for flag (CPU)."""

import os
import sys
from dataclasses import dataclass

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402

from dsb200.postproc import (HALO_DROPPED, TIME_EDGE_DROPPED, MergerConfig,  # noqa: E402
                             filter_to_canonical, merge_across_kernels, merge_across_kernels_c1)


@dataclass(frozen=True)
class Cand:
    l: float
    m: float
    dm_fine: float
    dm_idx: int
    event_specnum: int
    width_samples: int
    kernel_id: str
    snr: float
    flags: int


def _cands():
    l, m, d, t, w, snr, flags, kern = MG.postproc_fields()
    return [Cand(float(l[i]), float(m[i]), float(i), int(d[i]), int(t[i]), int(w[i]),
                 f"unit:d1:b{1 << int(kern[i])}", float(snr[i]), int(flags[i]))
            for i in range(len(l))]


def _ids(cs):
    return np.asarray([int(c.dm_fine) for c in cs], np.int64)


def test_mergers_match_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "postproc.npz"))
    cs = _cands()
    np.testing.assert_array_equal(_ids(merge_across_kernels_c1(cs, MergerConfig())),
                                  z["c1_default"])
    np.testing.assert_array_equal(
        _ids(merge_across_kernels_c1(cs, MergerConfig(lm_max_cells=5, dm_max_trials=1,
                                                      t_frac=0.5, sample_period_specnum=4))),
        z["c1_custom"])
    np.testing.assert_array_equal(_ids(merge_across_kernels(cs)), z["legacy"])
    np.testing.assert_array_equal(
        _ids(merge_across_kernels(cs, merge_radius_lm=2, merge_radius_fdm=3, merge_radius_t=50)),
        z["legacy_custom"])
    assert merge_across_kernels_c1([], MergerConfig()) == []
    with pytest.raises(ValueError):
        MergerConfig(lm_max_cells=-1)
    with pytest.raises(ValueError):
        merge_across_kernels(cs, merge_radius_t=-1)


def test_canonical_gate_matches_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "postproc.npz"))
    cs = _cands()
    emit, dropped = filter_to_canonical(cs, dm_idx_canonical_lo=5, dm_idx_canonical_hi=25,
                                        t_det=4000, n_kernel_max_t=128, cube_t_offset=100)
    np.testing.assert_array_equal(_ids(emit), z["emit"])
    np.testing.assert_array_equal(_ids(dropped), z["dropped"])
    np.testing.assert_array_equal([c.flags for c in dropped], z["dropped_flags"])
    assert all(c.flags & (HALO_DROPPED | TIME_EDGE_DROPPED) for c in dropped)
    assert all(e is cs[int(e.dm_fine)] for e in emit)
    with pytest.raises(ValueError):
        filter_to_canonical(cs, dm_idx_canonical_lo=3, dm_idx_canonical_hi=2, t_det=10,
                            n_kernel_max_t=2)
