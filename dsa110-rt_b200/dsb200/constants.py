"""Constants of the fast search path (src/dsart/common/constants.py).

The reference hard-wires its DSA-110 geometry; here those values are the
defaults of a parametric ``Band`` and of the kernel geometry arguments.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

NATIVE_SAMPLE_US = 32.768                 # constants.py:25
NTIMES_PER_PACKET = 2                     # samples per SNAP packet
NPACKETS_PER_BLOCK = 2048                 # fada page (constants.py:31)
NANTS = 96                                # constants.py:200
NPOL = 2
BADA_NPOL = 2
NCHAN_PER_CHGROUP = 384                   # constants.py:70
N_CHGROUP = 16                            # constants.py:67
K_DM_MS_GHZ2_PC = 4.148808                # constants.py:163
SPEED_OF_LIGHT_M_S = 299_792_458.0        # constants.py:178
PHI_LAT_OVRO_DEG = 37.234                 # constants.py:187
PHI_LAT_OVRO_RAD = math.radians(PHI_LAT_OVRO_DEG)
LEGACY_FLUFF_SCALE = 0.05                 # constants.py:373
T_INT_FAST_NATIVE = 8


def nbase_of(nants: int) -> int:
    return nants * (nants + 1) // 2


NBASE = nbase_of(NANTS)


@dataclass(frozen=True)
class Band:
    """Channelisation ``freq(g, c) = f0 - (ch0 + g*nchan + c) * dnu`` GHz,
    descending in frequency (constants.py:133-151, edge convention)."""

    n_chgroup: int = N_CHGROUP
    nchan: int = NCHAN_PER_CHGROUP
    f0_ghz: float = 1.530
    dnu_ghz: float = 0.250 / 8192
    ch0: int = 1024

    def freq_table(self) -> np.ndarray:
        g = np.arange(self.n_chgroup, dtype=np.int64)[:, None]
        c = np.arange(self.nchan, dtype=np.int64)[None, :]
        return self.f0_ghz - (self.ch0 + g * self.nchan + c).astype(np.float64) * self.dnu_ghz

    def summed_freq_table(self, csf: int) -> np.ndarray:
        """Band-centre of each ``csf`` group (coarse_dm/dm_plan.py:128-182)."""
        full = self.freq_table()
        if csf == 1:
            return full
        if self.nchan % csf:
            raise ValueError(f"chan_sum_factor={csf} does not divide nchan={self.nchan}")
        return full.reshape(self.n_chgroup, self.nchan // csf, csf).mean(axis=2)

    def chgroup_top(self) -> np.ndarray:
        return self.freq_table()[:, 0].copy()

    def bot_proc(self) -> float:
        return float(self.freq_table()[-1, -1])


DSA110_BAND = Band()


def band_from_edges(n_chgroup: int, nchan: int, f_top_ghz: float, f_bot_ghz: float) -> Band:
    """Band whose channel 0 upper edge is ``f_top`` and whose channel width
    puts ``n_chgroup*nchan`` channels across ``[f_bot, f_top]``."""
    n = n_chgroup * nchan
    return Band(n_chgroup=n_chgroup, nchan=nchan, f0_ghz=f_top_ghz,
                dnu_ghz=(f_top_ghz - f_bot_ghz) / n, ch0=0)
