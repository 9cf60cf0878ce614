"""DeterministicDetector on the library's fused detector kernel: the
production (streaming) form of the reference's detector
(detector/forward.py:512-1860; ``streaming=True``, the fused multi-boxcar
argmax path :1480-1620 and the end-of-cube Layer-2 update :1820-1835).

For one cube ``[T_det, N_fdm, H, W]`` the kernel bank's time boxcars (widths
1, 2, 4, ..., 2^L: the v1 collapsed bank of delta image kernels and d1 DM
kernels) are scored in one pass (``dsb_detect_sampled``): zero-prefixed
float32 padded cumsum along time, centred boxcars over the interior outputs
``[t_edge, T_det - t_edge)``, S/N = boxcar / sigma_k of the PREVIOUS cube,
the strict-'>' winner over the widths, compaction above the threshold.  The
same pass gathers each kernel's raw boxcar at its Layer-2 sample positions;
their clipped std updates the Layer-2 state for the next cube.  The decode
is decode_topk_argmax_lowmem's (top ``decoder_n_top * K`` by value, ties by
flat index, greedy merge radii); then the optional C1 merger, the
canonical-zone gate and the C1 emit floor.

Differences from the reference, stated: the Layer-2 sample positions are
drawn by a CPU generator seeded k (the reference draws on the cube's
device), at most 4096 per kernel (the reference default is 10^6; its
production configuration passes 10^5); banks with image kernels other than
the v1 deltas, DM boxcars wider than 1, or time widths that are not
1, 2, ..., 2^L raise NotImplementedError (the reference runs those through
its per-kernel unfused path).
"""

from __future__ import annotations

import math
from typing import List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .kernels import Kernel, build_kernel_bank
from .noise import Layer2State
from .postproc import filter_to_canonical, merge_across_kernels_c1
from .search import (Candidate, CandidateBuffer, Layer2Samples, _nms,
                     sigma_clipped_std_batched)

NOISE_WARMUP = 1 << 3                    # common/contracts.py:80
DEFAULT_MERGE_RADIUS_LM = 3              # detector/merger.py:206-212
DEFAULT_MERGE_RADIUS_FDM = 5
DEFAULT_MERGE_RADIUS_T = 128
CUBE_CADENCE_S_DEFAULT = 256 * 16 * 32.768 * 1e-6    # common/constants.py:533-548


class DeterministicDetector:
    """Streaming detector with the reference's constructor and forward
    surface (detector/forward.py:538-570, :891)."""

    def __init__(self, *, kernel_bank: Optional[Tuple[Kernel, ...]] = None,
                 threshold_sigma: float = 8.0, detector_version: str = "v1.M5",
                 device=None, dtype: torch.dtype = torch.float16,
                 merge_radius_lm: int = DEFAULT_MERGE_RADIUS_LM,
                 merge_radius_fdm: int = DEFAULT_MERGE_RADIUS_FDM,
                 merge_radius_t: int = DEFAULT_MERGE_RADIUS_T, merger_config=None,
                 c1_snr_min: Optional[float] = None, search_node_id: int = 0,
                 gpu_half: int = 0, cube_cadence_s: float = CUBE_CADENCE_S_DEFAULT,
                 layer2_tau_s: float = 30.0, layer2_n_burnin: int = 30,
                 n_kernel_max_t: Optional[int] = None, layer2_state: Optional[Layer2State] = None,
                 layer2_seed_unit: bool = True, layer2_sigma_floor: float = 0.0,
                 layer2_sigma_max_ratio: float = 0.0, layer2_clamp_escape_cubes: int = 0,
                 layer2_valid_min_fraction: float = 1.0, streaming: bool = True,
                 streaming_tile_size: int = 64, layer2_sigma_max_samples: Optional[int] = 4096,
                 streaming_decoder: str = "topk_lowmem", streaming_decoder_n_top: int = 64,
                 boxcar_accum_dtype=None, cand_capacity: int = 1 << 20):
        self.device = _lib.cuda_device(device if device is not None else "cuda")
        bank = kernel_bank if kernel_bank is not None else build_kernel_bank(
            ("unit",), ("d1",), ("b1", "b2", "b4", "b8", "b16", "b32", "b64"))
        if not bank:
            raise ValueError("kernel_bank is empty")
        widths = [int(k.k_time_width) for k in bank]
        if any(k.image_kernel_size != 1 or float(k.image_kernel.reshape(-1)[0]) != 1.0
               or k.k_dm_width != 1 for k in bank):
            raise NotImplementedError("only the collapsed bank (delta image kernels, d1) runs "
                                      "on the fused detector")
        logw = int(round(math.log2(max(widths))))
        if widths != [1 << i for i in range(logw + 1)] or logw > 6:
            raise NotImplementedError("the fused detector scores time widths 1, 2, ..., 2^L, "
                                      "L <= 6, in that order")
        if streaming_decoder != "topk_lowmem":
            raise NotImplementedError("only the topk_lowmem decoder is built")
        if not 0.0 <= layer2_valid_min_fraction <= 1.0:
            raise ValueError(f"layer2_valid_min_fraction={layer2_valid_min_fraction}, "
                             "expected in [0, 1]")
        if streaming_decoder_n_top < 1:
            raise ValueError(f"streaming_decoder_n_top={streaming_decoder_n_top}, expected ≥ 1")
        m = 4096 if layer2_sigma_max_samples is None else int(layer2_sigma_max_samples)
        if not 1 <= m <= 4096:
            raise ValueError("layer2_sigma_max_samples must be in [1, 4096] on this detector")
        self._bank = tuple(bank)
        self._widths = widths
        self._logw = logw
        self._threshold = float(threshold_sigma)
        self._detector_version = detector_version
        self._r = (int(merge_radius_lm), int(merge_radius_fdm), int(merge_radius_t))
        self._merger_config = merger_config
        self._c1_snr_min = c1_snr_min
        self._n_kernel_max_t = int(n_kernel_max_t) if n_kernel_max_t is not None else max(widths)
        self._m = m
        self._valid_min_fraction = float(layer2_valid_min_fraction)
        self._n_top = int(streaming_decoder_n_top)
        if layer2_state is None:
            layer2_state = Layer2State(len(bank), cube_cadence_s=cube_cadence_s,
                                       tau_s=layer2_tau_s, n_burnin=int(layer2_n_burnin),
                                       n_kernel_max_t=self._n_kernel_max_t,
                                       sigma_floor=float(layer2_sigma_floor),
                                       sigma_max_ratio=float(layer2_sigma_max_ratio),
                                       clamp_escape_cubes=int(layer2_clamp_escape_cubes),
                                       device=self.device)
            if layer2_seed_unit:
                # the analytic unit-noise value, sqrt(k_dm * k_time) (forward.py:746-755)
                layer2_state._s_k.copy_(torch.tensor(
                    [math.sqrt(k.k_dm_width * k.k_time_width) for k in bank],
                    dtype=layer2_state._s_k.dtype))
        self._layer2 = layer2_state
        self._cands = CandidateBuffer(self.device, cand_capacity)
        self._samples_key = None
        self._samples: Optional[Layer2Samples] = None
        self.spatial_active: Optional[torch.Tensor] = None

    # -- the reference's properties ---------------------------------------
    def kernels(self) -> Tuple[str, ...]:
        return tuple(k.kernel_id for k in self._bank)

    @property
    def kernel_bank(self) -> Tuple[Kernel, ...]:
        return self._bank

    @property
    def detector_version(self) -> str:
        return self._detector_version

    @property
    def threshold_sigma(self) -> float:
        return self._threshold

    @property
    def layer2_state(self) -> Layer2State:
        return self._layer2

    def set_spatial_active(self, spatial_active: Optional[torch.Tensor]) -> None:
        """Image cells inside the edge mask (1-D bool of length H*W): the
        Layer-2 samples outside it are dropped (forward.py:810-828)."""
        self.spatial_active = None if spatial_active is None else \
            torch.as_tensor(spatial_active).reshape(-1).to(torch.bool)
        self._samples_key = None

    def _cube_valid(self, validity_mask: torch.Tensor) -> bool:
        if self._valid_min_fraction >= 1.0:
            return bool(torch.all(validity_mask).item())
        n_total = int(validity_mask.numel())
        if n_total <= 0:
            return False
        return int(validity_mask.sum().item()) / n_total >= self._valid_min_fraction

    # -- forward -------------------------------------------------------------
    def forward(self, cube: torch.Tensor, validity_mask: torch.Tensor,
                sigma_layer1: torch.Tensor, *, dm_idx_canonical_lo: Optional[int] = None,
                dm_idx_canonical_hi: Optional[int] = None,
                n_kernel_max_t: Optional[int] = None, event_specnum: int = 0,
                fine_to_coarse=None, fine_dm_pc_cm3=None) -> List[Candidate]:
        """Candidates of one cube ``[T_det, N_fdm, H, W]`` (float16 or
        float32, on this detector's device); ``validity_mask [T_det, N_fdm]``
        bool decides whether the cube updates Layer-2; ``sigma_layer1`` is
        accepted for the reference's signature (the cube arrives already
        normalised, as in its streaming path)."""
        _lib.require_cuda(cube, "cube")
        if cube.dim() != 4:
            raise ValueError(f"cube.dim()={cube.dim()}, expected 4 [T_det, N_fdm, H, W]")
        if cube.dtype not in (torch.float16, torch.float32):
            raise ValueError(f"cube dtype {cube.dtype} not float16/float32")
        T, F, H, W = cube.shape
        if tuple(validity_mask.shape) != (T, F):
            raise ValueError(f"validity_mask shape {tuple(validity_mask.shape)}, expected {(T, F)}")
        if sigma_layer1 is not None and tuple(sigma_layer1.shape) != (F,):
            raise ValueError(f"sigma_layer1 shape {tuple(sigma_layer1.shape)}, expected {(F,)}")
        cube = cube.contiguous()
        K = len(self._bank)
        max_w = max(self._widths)
        if max_w > T:
            raise ValueError(f"widest boxcar {max_w} exceeds T_det={T}")
        nkmt = self._n_kernel_max_t if n_kernel_max_t is None else int(n_kernel_max_t)
        t_edge = max(0, nkmt // 2)
        t_base, n_out = (t_edge, T - 2 * t_edge) if t_edge > 0 and 2 * t_edge < T else (0, T)
        npix = H * W
        if npix % 256:
            raise ValueError("the fused detector needs H*W a multiple of 256")
        key = (T, F, npix, t_base, n_out)
        if self._samples_key != key:
            act = (np.ones(npix, bool) if self.spatial_active is None
                   else self.spatial_active.cpu().numpy())
            self._samples = Layer2Samples(n_kernels=K, m=self._m, n_out=n_out, n_fdm=F,
                                          npix=npix, active=act, device=self.device)
            self._samples_key = key
        l2 = self._samples
        cube_valid = self._cube_valid(validity_mask)
        sinv = torch.reciprocal(torch.clamp(self._layer2.s_k.to(self.device, torch.float32),
                                            min=1e-30)).contiguous()
        self._cands.reset()
        _lib.check(_lib.lib().dsb_detect_sampled(
            _lib.ptr(cube), int(cube.dtype == torch.float16), T, F, npix, npix, F * npix, None, 0,
            None, self._logw, _lib.ptr(sinv), t_base, n_out, self._threshold,
            _lib.ptr(self._cands.buf), self._cands.capacity, 0, _lib.ptr(self._cands.count),
            _lib.ptr(l2.d_off), _lib.ptr(l2.d_ent), _lib.ptr(l2.samples), l2.m,
            _lib.stream_of(self.device)), "dsb_detect_sampled")
        # decoder_n_top grows with the cube / interior ratio (forward.py:1383-1399)
        n_top = self._n_top
        if t_base > 0 and n_out < T:
            n_top = max(n_top, int(math.ceil(n_top * float(T) / float(n_out))))
        got = self._cands.fetch_top(n_top * K)
        items = [(float(c["snr"]), int(c["t"]) * (F * npix) + int(c["pix"]), int(c["k"]))
                 for c in got]
        r_lm, r_f, r_t = self._r
        dec = _nms(items, threshold=self._threshold, n_top=n_top * K, shape=(n_out, F, H, W),
                   r_t=r_t, r_f=r_f, r_lm=r_lm)
        f2c = None if fine_to_coarse is None else np.asarray(torch.as_tensor(fine_to_coarse).cpu())
        fdm = None if fine_dm_pc_cm3 is None else np.asarray(torch.as_tensor(fine_dm_pc_cm3).cpu())
        cands = [Candidate(l=float(l_), m=float(m_),
                           dm_fine=float(fdm[f]) if fdm is not None else float(f),
                           dm_idx=int(f2c[f]) if f2c is not None else int(f),
                           event_specnum=int(event_specnum) + t_base + int(t),
                           width_samples=self._widths[k], kernel_id=self._bank[k].kernel_id,
                           snr=float(v))
                 for t, f, l_, m_, v, k in dec]
        # end-of-cube Layer-2 update: the new sigma_k divides the next cube
        sig_k = sigma_clipped_std_batched(l2.samples)
        _, warming = self._layer2.update_and_query(per_kernel_sigma=sig_k, valid=cube_valid)
        if warming:
            cands = [Candidate(**{**c.__dict__, "flags": c.flags | NOISE_WARMUP}) for c in cands]
        if self._merger_config is not None:
            cands = merge_across_kernels_c1(cands, self._merger_config)
        if dm_idx_canonical_lo is not None and dm_idx_canonical_hi is not None:
            cands, _ = filter_to_canonical(cands, dm_idx_canonical_lo=dm_idx_canonical_lo,
                                           dm_idx_canonical_hi=dm_idx_canonical_hi, t_det=T,
                                           n_kernel_max_t=nkmt, cube_t_offset=event_specnum)
        if self._c1_snr_min is not None:
            cands = [c for c in cands if float(c.snr) >= float(self._c1_snr_min)]
        return cands

    __call__ = forward
