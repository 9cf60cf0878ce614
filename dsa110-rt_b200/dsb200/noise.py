"""Noise-state trackers of the detector's normalisation.

Layer-1 (noise_norm/layer1.py:342-600): per fine DM, a ring of the last
``n_burnin_cubes`` σ values; during the first ``n_burnin_cubes`` cubes the
σ used is the median of the ring so far, afterwards the cube's own σ; an
optional floor.

Layer-2 per-kernel noise state (noise_norm/layer2.py:113-452 of the
reference): one σ_k per detector kernel, a Welford running mean over the
first ``n_burnin`` cubes, then an EMA with γ = 1 − exp(−cube_cadence_s /
τ_s).  Each cube's σ_k estimate comes in through
``update_and_query(per_kernel_sigma=...)``; a zero estimate keeps the
previous value; ``sigma_max_ratio`` rejects an update above that multiple
of the previous σ_k unless the kernel has been rejected for
``clamp_escape_cubes`` cubes in a row (then σ_k rebaselines to the
estimate); ``sigma_floor`` (a scalar or one value per kernel) bounds σ_k
from below after the blend.

The state is a handful of float32 scalars per cube, updated with the same
tensor operations, in the same order, as the reference (so a state on the
same device type gives the same bits).  The estimate from a full
per-kernel score cube (``scores=``, the reference's
``layer2_interior_sigma``) is not built: the fused detector here never
materialises per-kernel score cubes; callers pass ``per_kernel_sigma``.
"""

from __future__ import annotations

import math
from collections import deque
from typing import Optional, Tuple

import numpy as np
import torch

NOISE_LAYER1_N_BURNIN_CUBES_DEFAULT = 5         # constants.py:556

T_INT_SEARCH_US_DEFAULT = 16 * 32.768         # constants.py:533
CUBE_CADENCE_S_DEFAULT = 256 * T_INT_SEARCH_US_DEFAULT * 1e-6   # constants.py:538-548
NOISE_LAYER2_TAU_S_DEFAULT = 30.0              # constants.py:564
NOISE_LAYER2_N_BURNIN_DEFAULT = 30             # constants.py:571
N_KERNEL_MAX_T_DEFAULT = 128                   # constants.py:550


class Layer1State:
    """Per-fine-DM Layer-1 σ with the cold-start burn-in (layer1.py:342)."""

    def __init__(self, n_fdm: int, *, n_burnin_cubes: int = NOISE_LAYER1_N_BURNIN_CUBES_DEFAULT,
                 sigma_floor: float = 0.0):
        if n_fdm < 1:
            raise ValueError(f"n_fdm={n_fdm}, expected ≥ 1")
        if n_burnin_cubes < 1:
            raise ValueError(f"n_burnin_cubes={n_burnin_cubes}, expected ≥ 1")
        if sigma_floor < 0.0:
            raise ValueError(f"sigma_floor={sigma_floor}, expected ≥ 0")
        self.n_fdm = int(n_fdm)
        self.n_burnin_cubes = int(n_burnin_cubes)
        self.sigma_floor = float(sigma_floor)
        self._history = [deque(maxlen=self.n_burnin_cubes) for _ in range(self.n_fdm)]
        self._cube_count = 0

    @property
    def cube_count(self) -> int:
        return self._cube_count

    @property
    def is_warming_up(self) -> bool:
        return self._cube_count < self.n_burnin_cubes

    def reset(self) -> None:
        for d in self._history:
            d.clear()
        self._cube_count = 0

    def update_and_query(self, cube: Optional[torch.Tensor] = None, *,
                         per_fdm_sigma: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Push this cube's per-fine-DM σ (``dsb200.search.layer1_sigma``
        computes it from the images) and return the σ to normalise this
        cube with (layer1.py:537-600)."""
        if cube is not None:
            raise NotImplementedError(
                "pass per_fdm_sigma (dsb200.search.layer1_sigma gathers it from the images)")
        if per_fdm_sigma is None:
            raise ValueError("pass exactly one of cube= or per_fdm_sigma=")
        sig = per_fdm_sigma.to(torch.float32)
        if sig.shape != (self.n_fdm,):
            raise ValueError(f"per-fdm sigma shape {tuple(sig.shape)} != (n_fdm={self.n_fdm},)")
        device = sig.device
        vals = sig.detach().cpu().numpy()
        for f in range(self.n_fdm):
            self._history[f].append(float(vals[f]))
        if self._cube_count < self.n_burnin_cubes:
            out = np.empty(self.n_fdm, dtype=np.float32)
            for f in range(self.n_fdm):
                out[f] = float(np.median(list(self._history[f])))
            self._cube_count += 1
            out_t = torch.from_numpy(out).to(device)
        else:
            self._cube_count += 1
            out_t = sig
        if self.sigma_floor > 0.0:
            out_t = out_t.clamp_min(float(self.sigma_floor))
        return out_t


class Layer2State:
    """Per-kernel σ_k tracker: Welford burn-in, then EMA (layer2.py:113)."""

    def __init__(self, n_kernels: int, *, cube_cadence_s: float = CUBE_CADENCE_S_DEFAULT,
                 tau_s: float = NOISE_LAYER2_TAU_S_DEFAULT,
                 n_burnin: int = NOISE_LAYER2_N_BURNIN_DEFAULT,
                 n_kernel_max_t: int = N_KERNEL_MAX_T_DEFAULT, sigma_floor=0.0,
                 sigma_max_ratio: float = 0.0, clamp_escape_cubes: int = 0,
                 device: Optional[torch.device] = None, dtype: torch.dtype = torch.float32):
        if n_kernels < 1:
            raise ValueError(f"n_kernels={n_kernels}, expected ≥ 1")
        if tau_s <= 0:
            raise ValueError(f"tau_s={tau_s}, expected > 0")
        if cube_cadence_s <= 0:
            raise ValueError(f"cube_cadence_s={cube_cadence_s}, expected > 0")
        if n_burnin < 0:
            raise ValueError(f"n_burnin={n_burnin}, expected ≥ 0")
        if n_kernel_max_t < 1:
            raise ValueError(f"n_kernel_max_t={n_kernel_max_t}, expected ≥ 1")
        floor_vec = None
        if isinstance(sigma_floor, (list, tuple)) or getattr(sigma_floor, "ndim", 0) > 0:
            floor_vec = torch.as_tensor(sigma_floor, dtype=dtype, device=device).reshape(-1)
            if floor_vec.numel() != int(n_kernels):
                raise ValueError(f"per-kernel sigma_floor has {floor_vec.numel()} entries, "
                                 f"expected n_kernels={n_kernels}")
            if bool((floor_vec < 0).any()):
                raise ValueError("per-kernel sigma_floor must be >= 0")
            sigma_floor = float(floor_vec.min())
        if float(sigma_floor) < 0:
            raise ValueError(f"sigma_floor={sigma_floor}, expected ≥ 0")
        if sigma_max_ratio < 0:
            raise ValueError(f"sigma_max_ratio={sigma_max_ratio}, expected ≥ 0")
        if clamp_escape_cubes < 0:
            raise ValueError(f"clamp_escape_cubes={clamp_escape_cubes}, expected ≥ 0")
        self.n_kernels = int(n_kernels)
        self.cube_cadence_s = float(cube_cadence_s)
        self.tau_s = float(tau_s)
        self.n_burnin = int(n_burnin)
        self.n_kernel_max_t = int(n_kernel_max_t)
        self.sigma_floor = float(sigma_floor)
        self._floor_vec = floor_vec
        self.sigma_max_ratio = float(sigma_max_ratio)
        self.clamp_escape_cubes = int(clamp_escape_cubes)
        self.gamma = 1.0 - math.exp(-self.cube_cadence_s / self.tau_s)
        self._s_k = torch.ones((self.n_kernels,), dtype=dtype, device=device)
        self._cube_count = 0
        i64 = dict(dtype=torch.int64, device=device)
        self._n_clamped = 0
        self._clamped = torch.zeros((self.n_kernels,), **i64)
        self._streak = torch.zeros((self.n_kernels,), **i64)
        self._n_escapes = 0
        self._escapes = torch.zeros((self.n_kernels,), **i64)

    # -- queries ---------------------------------------------------------
    @property
    def s_k(self) -> torch.Tensor:
        return self._s_k.detach().clone()

    @property
    def cube_count(self) -> int:
        return self._cube_count

    @property
    def is_warming_up(self) -> bool:
        return self._cube_count < self.n_burnin

    @property
    def n_clamped_high(self) -> int:
        return int(self._n_clamped)

    @property
    def per_kernel_clamped_high(self) -> torch.Tensor:
        return self._clamped.detach().clone()

    @property
    def n_clamp_escapes(self) -> int:
        return int(self._n_escapes)

    @property
    def per_kernel_clamp_escapes(self) -> torch.Tensor:
        return self._escapes.detach().clone()

    @property
    def per_kernel_clamp_streak(self) -> torch.Tensor:
        return self._streak.detach().clone()

    def reset(self) -> None:
        self._s_k.fill_(1.0)
        self._cube_count = 0
        self._n_clamped = 0
        self._clamped.zero_()
        self._streak.zero_()
        self._n_escapes = 0
        self._escapes.zero_()

    # -- update ----------------------------------------------------------
    def update_and_query(self, scores: Optional[torch.Tensor] = None, *,
                         per_kernel_sigma: Optional[torch.Tensor] = None,
                         valid: bool = True) -> Tuple[torch.Tensor, bool]:
        """Fold one cube's per-kernel σ estimate in and return ``(s_k,
        is_warming_up)`` after the update (layer2.py:313-452).  An invalid
        cube (``valid=False``) leaves the state untouched."""
        if scores is not None:
            raise NotImplementedError(
                "per-kernel score cubes are not materialised by this detector; "
                "pass per_kernel_sigma")
        if per_kernel_sigma is None:
            raise ValueError("pass exactly one of scores= or per_kernel_sigma=")
        if not valid:
            return self._s_k.detach().clone(), self.is_warming_up
        sig = per_kernel_sigma.to(self._s_k.dtype).to(self._s_k.device)
        if sig.shape != (self.n_kernels,):
            raise ValueError(f"per-kernel sigma shape {tuple(sig.shape)} != "
                             f"(n_kernels={self.n_kernels},)")
        zero = sig == 0
        if torch.any(zero):
            sig = torch.where(zero, self._s_k, sig)
        if self.sigma_max_ratio > 0.0 and self._cube_count > 0:
            high = sig > self.sigma_max_ratio * self._s_k
            if torch.any(high):
                if self.clamp_escape_cubes > 0:
                    escape = high & (self._streak >= self.clamp_escape_cubes)
                else:
                    escape = torch.zeros_like(high)
                clamp = high & ~escape
                if torch.any(escape):
                    self._s_k = torch.where(escape, sig, self._s_k)
                    self._escapes += escape.to(self._escapes.dtype)
                    self._n_escapes += int(escape.sum().item())
                if torch.any(clamp):
                    sig = torch.where(clamp, self._s_k, sig)
                    self._clamped += clamp.to(self._clamped.dtype)
                    self._n_clamped += int(clamp.sum().item())
                self._streak = torch.where(clamp, self._streak + 1,
                                           torch.zeros_like(self._streak))
            else:
                self._streak.zero_()
        if self._cube_count < self.n_burnin:
            count = float(self._cube_count)
            self._s_k = (count * self._s_k + sig) / (count + 1.0)
        else:
            self._s_k = self.gamma * sig + (1.0 - self.gamma) * self._s_k
        if self._floor_vec is not None:
            self._s_k = torch.maximum(self._s_k, self._floor_vec.to(self._s_k.device))
        elif self.sigma_floor > 0.0:
            self._s_k = torch.clamp(self._s_k, min=self.sigma_floor)
        self._cube_count += 1
        return self._s_k.detach().clone(), self.is_warming_up
