"""The detector's kernel bank (detector/kernels.py:85-300 of the reference).

A kernel is one (image, DM, time) token triple, ``"<image>:<dm>:<time>"``:
the image kernel (``unit``, ``psf``, ``psf_shift_lm``, ``psf_shift_l``; all
1 x 1 deltas of weight 1 in the reference's v1 detector), a centred DM
boxcar of odd width (``d1``..``d7``, fine-DM bins) and a time boxcar of
power-of-two width (``b1``..``b128``, search samples).  The bank is the
Cartesian product in (image, dm, time) order, so kernel k's flat index is
``i_img * n_dm * n_time + i_dm * n_time + i_time``; the Layer-2 state and
the decoder's kernel ids use that order.  The records and their
validation are the reference's interface; the boxcars themselves are the
library's detector kernels.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence, Tuple

import torch

DETECTOR_K_TIME_WIDTHS: Tuple[int, ...] = (1, 2, 4, 8, 16, 32, 64, 128)   # constants.py:274
DETECTOR_K_DM_WIDTHS: Tuple[int, ...] = (1, 3, 5, 7)                      # constants.py:277
DETECTOR_IMAGE_KERNELS: Tuple[str, ...] = ("unit", "psf", "psf_shift_lm", "psf_shift_l")
DETECTOR_DM_KERNELS: Tuple[str, ...] = tuple(f"d{w}" for w in DETECTOR_K_DM_WIDTHS)
DETECTOR_TIME_KERNELS: Tuple[str, ...] = tuple(f"b{w}" for w in DETECTOR_K_TIME_WIDTHS)
DEFAULT_DETECTOR_DTYPE: torch.dtype = torch.float16


@dataclass(frozen=True)
class Kernel:
    """One kernel triple (kernels.py:85-118)."""
    kernel_id: str
    image_token: str
    dm_token: str
    time_token: str
    k_dm_width: int
    k_time_width: int
    image_kernel: torch.Tensor
    image_kernel_size: int


def make_image_kernel(image_token: str, *, dtype: torch.dtype = DEFAULT_DETECTOR_DTYPE
                      ) -> torch.Tensor:
    """The image-axis kernel of a token: every v1 token is the 1 x 1 delta
    (weight 1, L1-normalised) (kernels.py:132-175)."""
    if image_token not in DETECTOR_IMAGE_KERNELS:
        raise ValueError(f"image_token={image_token!r} not in {DETECTOR_IMAGE_KERNELS}")
    return torch.ones((1, 1), dtype=dtype)


def _parse_width(token: str) -> int:
    if not token or token[0] not in ("d", "b") or not token[1:].isdigit():
        raise ValueError(f"token {token!r} not of form 'd<int>' or 'b<int>'")
    return int(token[1:])


def build_kernel_bank(image_tokens: Sequence[str] = DETECTOR_IMAGE_KERNELS,
                      dm_tokens: Sequence[str] = DETECTOR_DM_KERNELS,
                      time_tokens: Sequence[str] = DETECTOR_TIME_KERNELS, *,
                      dtype: torch.dtype = DEFAULT_DETECTOR_DTYPE) -> Tuple[Kernel, ...]:
    """The bank ``image_tokens x dm_tokens x time_tokens`` in (image, dm,
    time) order (kernels.py:191-300), with the reference's checks: tokens
    from the closed sets, DM widths odd, time widths powers of two."""
    for tok in image_tokens:
        if tok not in DETECTOR_IMAGE_KERNELS:
            raise ValueError(f"image_token {tok!r} not in {DETECTOR_IMAGE_KERNELS}")
    for tok in dm_tokens:
        if tok not in DETECTOR_DM_KERNELS:
            raise ValueError(f"dm_token {tok!r} not in {DETECTOR_DM_KERNELS}")
    for tok in time_tokens:
        if tok not in DETECTOR_TIME_KERNELS:
            raise ValueError(f"time_token {tok!r} not in {DETECTOR_TIME_KERNELS}")
    bank = []
    for it in image_tokens:
        ik = make_image_kernel(it, dtype=dtype)
        for dt in dm_tokens:
            k_dm = _parse_width(dt)
            if k_dm not in DETECTOR_K_DM_WIDTHS:
                raise ValueError(f"dm_token {dt!r} parses to width {k_dm}, not in "
                                 f"{DETECTOR_K_DM_WIDTHS}")
            if k_dm % 2 == 0:
                raise ValueError(f"dm_token {dt!r}: K_dm width must be odd (centred boxcar); "
                                 f"got {k_dm}")
            for tt in time_tokens:
                k_t = _parse_width(tt)
                if k_t not in DETECTOR_K_TIME_WIDTHS:
                    raise ValueError(f"time_token {tt!r} parses to width {k_t}, not in "
                                     f"{DETECTOR_K_TIME_WIDTHS}")
                if k_t & (k_t - 1):
                    raise ValueError(f"time_token {tt!r}: K_time width must be a power of two; "
                                     f"got {k_t}")
                bank.append(Kernel(kernel_id=f"{it}:{dt}:{tt}", image_token=it, dm_token=dt,
                                   time_token=tt, k_dm_width=k_dm, k_time_width=k_t,
                                   image_kernel=ik, image_kernel_size=int(ik.shape[-1])))
    return tuple(bank)
