"""Wire encoding of dedispersed rows on the device.

``encode_rows`` mirrors ``TransportTx._encode_rows``
(src/dsart/transport/tx.py:825-873): one DM row of ``n_fv`` tiles,
``(n_fv, n_filled)`` complex, is encoded tile by tile.

* ``BITS_CINT8_COMPLEX`` (16 bits per cell): cint8 with a per-tile scale,
  ``amax / 127``;
* ``BITS_CFP16_COMPLEX`` (32 bits per cell): half-precision parts, scale 1.

The result is the same (bit for bit) as the reference's.  Here it stays on
the device: ``(payloads, scales)`` with payloads ``(n_fv, n_filled, 2)``
int8 or float16, and scales ``(n_fv,)`` float32.
"""

from __future__ import annotations

import torch

from . import _lib

BITS_CINT8_COMPLEX = 16
BITS_CFP16_COMPLEX = 32


def encode_rows(row: torch.Tensor, bits_per_cell: int):
    """Encode all tiles of one DM row ``(n_fv, n_filled)`` complex64 (CUDA);
    tiles may be strided (a view of every k-th tile), cells must be dense."""
    if not isinstance(row, torch.Tensor) or row.device.type != "cuda":
        raise ValueError("row must be a CUDA tensor (dsb200 has no CPU path)")
    if row.dim() != 2:
        raise ValueError(f"row must be (n_fv, n_filled); got {tuple(row.shape)}")
    if bits_per_cell not in (BITS_CINT8_COMPLEX, BITS_CFP16_COMPLEX):
        raise AssertionError(f"unhandled bits_per_cell={bits_per_cell}")
    row = row.to(torch.complex64)
    if row.stride(1) != 1:
        row = row.contiguous()
    n_fv, n_filled = row.shape
    dt = torch.int8 if bits_per_cell == BITS_CINT8_COMPLEX else torch.float16
    payload = torch.empty((n_fv, n_filled, 2), dtype=dt, device=row.device)
    scales = torch.empty(n_fv, dtype=torch.float32, device=row.device)
    _lib.check(_lib.lib().dsb_encode_rows(_lib.ptr(row), row.stride(0) if n_fv else n_filled,
                                          n_fv, n_filled, bits_per_cell, _lib.ptr(payload),
                                          _lib.ptr(scales), _lib.stream_of(row.device)),
               "dsb_encode_rows")
    return payload, scales
